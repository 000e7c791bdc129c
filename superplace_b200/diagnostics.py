"""GP diagnostics (the reference's --gp-diagnostics) from the device engine.

writeGpDiagnostic and diagnoseDelivered (src/gp/diagnostics.h:13-23, src/gp/diagnostics.cpp:39-191)
write, for one evaluation point of a GP stage, into <root>/diagnostics/<stage>/<point>/:

  bins.csv      every bin: its rectangle, capacity, the four charge maps, overflow area (with and
                without the movable nodes), potential, field and overflow component;
  nodes.csv     every opt node: position, size, WA gradient, density force, preconditioner,
                gradient, movement since the previous evaluation, the component it overlaps most;
  geometry.csv  the fixed nodes and the site rows;
  metadata.json the point's lambda, gamma and step, the grid, the overflow and energy, the
                connected overflow components, and six probes (the overflow and energy after a
                small move of the opt nodes along the density direction and along the gradient).

EPlace::run writes them at first_eval (iteration 0), stagnation_mid (when the stagnation counter
first reaches half its window), last_eval and delivered (eplace.cpp:284-288,365-369,428-433,
476-479,505-507), for mGP and cGP. Here the device loop pauses at those points (the iteration and
stagnation callbacks of include/spgpu.h) and the maps, field, gradient and force are evaluated on
a copy of the PlaceDB at the handed positions, as the reference's probes run on deep copies: the
running stage is never touched. Numbers are written as the reference's streams write them
(std::setprecision(17) in the CSV files; nlohmann::json, keys sorted, in metadata.json).
"""
from __future__ import annotations

import json
import os

import numpy as np

from . import abi, engine
from .metrics import STAGE_NAMES
from .placedb import F_FILLER, F_FIXED, F_MACRO, F_NI, PlaceDB

f32 = np.float32


def g17(v) -> str:
    """A float or double as the reference's stream writes it with std::setprecision(17)."""
    return format(float(v), ".17g")


def opt_index(db: PlaceDB, stage: int) -> np.ndarray:
    """EPlace::Impl::buildOptSet (src/gp/eplace.cpp:82-94): the stage's movable cells (no fixed,
    no NI; cGP also leaves the macros out; FILLERONLY has none), then every filler."""
    fl = db.node_flags[: db.num_movable]
    cells = np.zeros(0, np.int64)
    if stage != abi.STAGE_FILLER_ONLY:
        keep = (fl & (F_FIXED | F_NI)) == 0
        if stage == abi.STAGE_CGP:
            keep &= (fl & F_MACRO) == 0
        cells = np.nonzero(keep)[0]
    return np.concatenate([cells, np.arange(db.num_nodes, db.total_nodes)]).astype(np.int64)


def compute_gamma(tau: float, bin_step: float) -> float:
    """computeGamma (src/gp/wa_wirelength.cpp:18-29) in float arithmetic."""
    gamma = f32(8.0) * f32(bin_step)
    tau = f32(tau)
    if tau > f32(1.0):
        gamma = f32(gamma * f32(10.0))
    elif tau < f32(0.1):
        gamma = f32(gamma * f32(0.1))
    else:
        gamma = f32(gamma * np.power(f32(10.0), f32(f32(f32(20.0) / f32(9.0)) * f32(tau - f32(0.1))) - f32(1.0)))
    return float(max(gamma, f32(1e-4)))


class Evaluation:
    """One evaluation of the density and wirelength operators at given positions on a copy of
    the PlaceDB (its own device context): the maps, field, WA gradient and density force."""

    def __init__(self, db: PlaceDB, params: abi.Params, dim: int):
        self.db = db.copy()
        self.params = params
        self.dim = dim
        self.ctx = engine.GpContext(self.db, params)

    def close(self):
        self.ctx.close()

    def at(self, x, y, gamma=None):
        """Evaluate at node positions (x, y): the grid rebuilt, the charge accumulated and the
        field solved (BinGrid::initialize, accumulate, solveField); with gamma also the WA
        gradient and the density force (WaWirelength::compute, BinGrid::gatherForce)."""
        db, ctx = self.db, self.ctx
        db.node_x[:] = x
        db.node_y[:] = y
        ctx.set_positions(db.node_x, db.node_y)
        ctx.set_flags(db.node_flags)
        info = ctx.grid_init(self.params.target_density, self.dim)
        ctx.accumulate()
        tau = ctx.overflow()  # also forms the float maps and rho from the fixed-point charge
        ctx.solve_field()
        maps = {k: ctx.read_map(w) for k, w in (("node", 0), ("filler", 1), ("terminal", 2), ("base", 3),
                                                   ("phi", 5), ("ex", 6), ("ey", 7))}
        out = dict(info=info, maps=maps, overflow=tau)
        if gamma is not None:
            _, out["wl_grad"] = ctx.wa(gamma, self.params.ignore_net_degree)
            out["force"] = ctx.gather_force()
        return out


def _footprints(db, x, y, idx, g):
    """BinGrid::footprintOf (src/gp/bin_grid.cpp:22-53) of nodes idx at positions x, y: the
    smoothed rectangle and the bin range, in the reference's float operations."""
    sx, sy, ox, oy, dim = f32(g["step_x"]), f32(g["step_y"]), f32(g["origin_x"]), f32(g["origin_y"]), g["dim"]
    w, h = db.node_w[idx], db.node_h[idx]
    cx, cy = x[idx], y[idx]
    half = f32(0.5)
    lx, hx = cx - half * w, cx + half * w
    ly, hy = cy - half * h, cy + half * h
    nx, ny = w < sx, h < sy
    lx = np.where(nx, cx - half * sx, lx)
    hx = np.where(nx, cx + half * sx, hx)
    ly = np.where(ny, cy - half * sy, ly)
    hy = np.where(ny, cy + half * sy, hy)

    def index(a, o, s):
        return np.clip(np.trunc((a - o) / s).astype(np.int64), 0, dim - 1)

    return (lx.astype(f32), ly.astype(f32), hx.astype(f32), hy.astype(f32),
            index(lx, ox, sx), index(hx, ox, sx), index(ly, oy, sy), index(hy, oy, sy))


def _bin_overlap(g, bx, by, lx, ly, hx, hy):
    """overlapArea(rect, bin) (src/db/geometry.h:35-39) with the bin's corners formed as
    originX + x * stepX (diagnostics.cpp:120-123), in float."""
    sx, sy, ox, oy = f32(g["step_x"]), f32(g["step_y"]), f32(g["origin_x"]), f32(g["origin_y"])
    blx = ox + bx.astype(f32) * sx
    bly = oy + by.astype(f32) * sy
    dx = np.minimum(hx, blx + sx) - np.maximum(lx, blx)
    dy = np.minimum(hy, bly + sy) - np.maximum(ly, bly)
    return np.where((dx > 0) & (dy > 0), dx * dy, f32(0.0)).astype(f32)


def _components(excess, dim):
    """The connected overflow components (4-neighbour, bins with positive excess) in the
    reference's order: ids by first bin in scan order, each grown breadth first from it, its
    overflow area summed in visiting order (diagnostics.cpp:45-72)."""
    labels = np.full(dim * dim, -1, np.int64)
    comps = []
    pos = np.nonzero(excess > 0)[0]
    for b in pos:
        if labels[b] >= 0:
            continue
        cid = len(comps)
        queue = [int(b)]
        labels[b] = cid
        mass = 0.0
        mnx = mny = dim
        mxx = mxy = 0
        h = 0
        while h < len(queue):
            here = queue[h]
            h += 1
            xx, yy = divmod(here, dim)
            mass += float(excess[here])
            mnx, mxx, mny, mxy = min(mnx, xx), max(mxx, xx), min(mny, yy), max(mxy, yy)
            for q in (here - dim if xx > 0 else -1, here + dim if xx + 1 < dim else -1,
                      here - 1 if yy > 0 else -1, here + 1 if yy + 1 < dim else -1):
                if q >= 0 and labels[q] < 0 and excess[q] > 0:
                    labels[q] = cid
                    queue.append(q)
        comps.append({"id": cid, "bins": len(queue), "overflow_area": mass, "bin_bounds": [mnx, mny, mxx, mxy]})
    return labels, comps


def _node_components(db, x, y, idx, g, labels):
    """The component each opt node overlaps most (diagnostics.cpp:106-119): per component the
    node's overlap areas with its labelled footprint bins, summed in bin order; the largest
    positive sum, ties to the smaller id; -1 without one."""
    dim = g["dim"]
    lx, ly, hx, hy, bx0, bx1, by0, by1 = _footprints(db, x, y, idx, g)
    spx, spy = bx1 - bx0 + 1, by1 - by0 + 1
    out = np.full(idx.size, -1, np.int64)
    small = (spx <= 4) & (spy <= 4)
    s = np.nonzero(small)[0]
    lab, wt = [], []
    for a in range(4):
        for b in range(4):
            ok = (a < spx[s]) & (b < spy[s])
            bx, by = np.minimum(bx0[s] + a, dim - 1), np.minimum(by0[s] + b, dim - 1)
            L = np.where(ok, labels[bx * dim + by], -1)
            W = np.where(L >= 0, _bin_overlap(g, bx, by, lx[s], ly[s], hx[s], hy[s]).astype(np.float64), 0.0)
            lab.append(L)
            wt.append(W)
    best_t = np.zeros(s.size)
    best_l = np.full(s.size, -1, np.int64)
    for j in range(len(lab)):
        Lj = lab[j]
        t = np.zeros(s.size)
        for k in range(len(lab)):  # the label's sum in bin order
            t = t + np.where(lab[k] == Lj, wt[k], 0.0)
        better = (Lj >= 0) & (t > 0) & ((t > best_t) | ((t == best_t) & (Lj < best_l)))
        best_t = np.where(better, t, best_t)
        best_l = np.where(better, Lj, best_l)
    out[s] = best_l
    for k in np.nonzero(~small)[0]:  # large footprints, one by one
        weights = {}
        for bx in range(bx0[k], bx1[k] + 1):
            bys = np.arange(by0[k], by1[k] + 1)
            L = labels[bx * dim + bys]
            if not np.any(L >= 0):
                continue
            W = _bin_overlap(g, np.full(bys.size, bx), bys, lx[k], ly[k], hx[k], hy[k])
            for lb, wv in zip(L, W):
                if lb >= 0:
                    weights[int(lb)] = weights.get(int(lb), 0.0) + float(wv)
        comp, most = -1, 0.0
        for cid in sorted(weights):
            if weights[cid] > most:
                comp, most = cid, weights[cid]
        out[k] = comp
    return out


def _energy(m):
    """energy(grid) (diagnostics.cpp:30-36): sum of 0.5 (node + filler + terminal + base) phi
    over the bins, in bin order."""
    q = ((m["node"].astype(np.float64) + m["filler"]) + m["terminal"]) + m["base"]
    return float(np.cumsum((0.5 * q * m["phi"]).ravel())[-1])


def _excess(m, target, bin_area, static_only=False):
    """excess(grid, b) (diagnostics.cpp:24-29) of every bin."""
    q = m["terminal"].astype(np.float64) + m["base"]
    if not static_only:
        q = q + m["node"]
    return np.maximum(0.0, q - float(target) * float(bin_area)).ravel()


def write_gp_diagnostic(root, stage, point, it, lam, gamma, step, db, params, dim, x, y, previous=None,
                        evaluation: Evaluation | None = None):
    """writeGpDiagnostic (src/gp/diagnostics.cpp:39-172) for the evaluation point (x, y) of
    node positions (every node) of `stage`, evaluated with lambda `lam` and gamma `gamma`;
    `previous` = the opt nodes' positions (x then y, opt order) at the evaluation before, or
    None at the first. The maps, field, WA gradient and force are evaluated at (x, y) on a copy
    of db (`evaluation`, created when not given). Returns the directory written."""
    name = STAGE_NAMES[stage]
    out_dir = os.path.join(root, "diagnostics", name, point)
    os.makedirs(out_dir, exist_ok=True)
    own = evaluation is None
    ev = Evaluation(db, params, dim) if own else evaluation
    try:
        x = np.ascontiguousarray(x, f32)
        y = np.ascontiguousarray(y, f32)
        e = ev.at(x, y, gamma)
        g, m = e["info"], e["maps"]
        dim = g["dim"]
        sx, sy = f32(g["step_x"]), f32(g["step_y"])
        bin_area = f32(sx * sy)
        target = f32(params.target_density)
        exc = _excess(m, target, bin_area)
        exc_static = _excess(m, target, bin_area, True)
        labels, comps = _components(exc, dim)
        overflow_area = float(np.cumsum(exc)[-1]) if exc.size else 0.0
        static_area = float(np.cumsum(exc_static)[-1]) if exc.size else 0.0
        _write_bins(out_dir, g, m, target, bin_area, exc, exc_static, labels)
        idx = opt_index(db, stage)
        dens, comb = _write_nodes(out_dir, db, x, y, idx, g, labels, f32(lam), e["wl_grad"], e["force"], previous)
        _write_geometry(out_dir, db, x, y)
        probes = _probes(ev, db, params, x, y, idx, g, dens, comb)
        denom = float(g["overflow_denominator"])
        meta = {"stage": name, "point": point, "iter": int(it),
                "movement_reference": ("last evaluation (includes rollback jump)" if point == "delivered"
                                       else "previous evaluation"),
                "eval_lambda": float(f32(lam)), "eval_gamma": float(f32(gamma)), "step_size": float(f32(step)),
                "grid_dim": int(dim), "origin": [float(f32(g["origin_x"])), float(f32(g["origin_y"]))],
                "bin_step": [float(sx), float(sy)], "overflow_denominator": denom,
                "overflow_area": overflow_area, "overflow": float(f32(e["overflow"])),
                "static_overflow_area": static_area, "static_floor_tau": static_area / denom if denom > 0 else 0.0,
                "energy": _energy(m), "components": comps, "probes": probes}
        with open(os.path.join(out_dir, "metadata.json"), "w") as f:
            f.write(json.dumps(meta, indent=2, sort_keys=True) + "\n")
    finally:
        if own:
            ev.close()
    return out_dir


def _csv(path, header, cols):
    """One CSV file: the header, then one line per row of the columns (strings or numbers)."""
    def text(c):
        if isinstance(c, np.ndarray) and c.dtype.kind == "f":
            return [g17(v) for v in c.tolist()]
        if isinstance(c, np.ndarray):
            return [str(v) for v in c.tolist()]
        return c
    cols = [text(c) for c in cols]
    with open(path, "w") as f:
        f.write(header + "\n")
        f.writelines(",".join(r) + "\n" for r in zip(*cols))


def _write_bins(out_dir, g, m, target, bin_area, exc, exc_static, labels):
    dim = g["dim"]
    sx, sy, ox, oy = f32(g["step_x"]), f32(g["step_y"]), f32(g["origin_x"]), f32(g["origin_y"])
    bx, by = np.divmod(np.arange(dim * dim), dim)
    lx = ox + bx.astype(f32) * sx
    ly = oy + by.astype(f32) * sy
    cap = np.full(dim * dim, float(target) * float(bin_area))
    _csv(os.path.join(out_dir, "bins.csv"),
         "bx,by,lx,ly,hx,hy,capacity,node_charge,filler_charge,terminal_charge,base_charge,overflow_area,"
         "static_overflow_area,potential,field_x,field_y,component",
         [bx, by, lx, ly, (lx + sx).astype(f32), (ly + sy).astype(f32), cap, m["node"].ravel(), m["filler"].ravel(),
          m["terminal"].ravel(), m["base"].ravel(), exc, exc_static, m["phi"].ravel(), m["ex"].ravel(),
          m["ey"].ravel(), labels])


def _write_nodes(out_dir, db, x, y, idx, g, labels, lam, wl_grad, force, previous):
    """nodes.csv (diagnostics.cpp:101-144); returns the density and combined directions."""
    n, total, nm = idx.size, db.total_nodes, db.num_movable
    comp = _node_components(db, x, y, idx, g, labels)
    mov = idx < nm
    wx = np.where(mov, wl_grad[np.minimum(idx, max(nm - 1, 0))], f32(0)).astype(f32) if nm else np.zeros(n, f32)
    wy = np.where(mov, wl_grad[nm + np.minimum(idx, max(nm - 1, 0))], f32(0)).astype(f32) if nm else np.zeros(n, f32)
    fx, fy = force[idx].astype(f32), force[total + idx].astype(f32)
    deg = np.diff(db.node2pin_start)[idx].astype(np.float64)
    area = db.node_w[idx].astype(np.float64) * db.node_h[idx].astype(np.float64)
    pre = (1.0 / np.maximum(1.0, deg + float(lam) * area)).astype(f32)
    lfx, lfy = (lam * fx).astype(f32), (lam * fy).astype(f32)
    gx, gy = (pre * (wx - lfx)).astype(f32), (pre * (wy - lfy)).astype(f32)
    dens = np.concatenate([(pre * lam).astype(f32) * fx, (pre * lam).astype(f32) * fy]).astype(f32)
    comb = np.concatenate([-gx, -gy]).astype(f32)
    px, py = x[idx], y[idx]
    if previous is not None and len(previous) == 2 * n:
        prev = np.asarray(previous, f32)
        dx = px.astype(np.float64) - prev[:n]
        dy = py.astype(np.float64) - prev[n:]
    else:
        dx = dy = np.zeros(n)
    w, h = db.node_w[idx], db.node_h[idx]
    half, eps = f32(0.5), f32(0.01)
    clx, cly, chx, chy = (f32(v) for v in db.core)
    boundary = ((px - half * w <= clx + eps) | (py - half * h <= cly + eps) |
                (px + half * w >= chx - eps) | (py + half * h >= chy - eps)).astype(np.int64)
    names = getattr(db, "node_names", None)
    quoted = ['"' + (names[i] if names is not None else "o%d" % i).replace('"', '""') + '"' for i in idx.tolist()]
    fl = db.node_flags[idx]
    _csv(os.path.join(out_dir, "nodes.csv"),
         "id,name,filler,macro,component,x,y,width,height,wl_x,wl_y,force_x,force_y,lambda_force_x,"
         "lambda_force_y,preconditioner,gradient_x,gradient_y,actual_dx,actual_dy,boundary",
         [idx, quoted, ((fl & F_FILLER) != 0).astype(np.int64), ((fl & F_MACRO) != 0).astype(np.int64), comp,
          px, py, w, h, wx, wy, fx, fy, lfx, lfy, pre, gx, gy, dx, dy, boundary])
    return dens, comb


def _write_geometry(out_dir, db, x, y):
    """geometry.csv (diagnostics.cpp:145-153): fixed non-NI nodes, then the site rows."""
    half = f32(0.5)
    fl = db.node_flags[: db.num_nodes]
    fixed = np.nonzero(((fl & F_FIXED) != 0) & ((fl & F_NI) == 0))[0]
    w, h = db.node_w[fixed], db.node_h[fixed]
    lines = ["kind,id,lx,ly,hx,hy"]
    for i, a, b, c, d in zip(fixed.tolist(), (x[fixed] - half * w).tolist(), (y[fixed] - half * h).tolist(),
                             (x[fixed] + half * w).tolist(), (y[fixed] + half * h).tolist()):
        lines.append(f"fixed,{i},{g17(a)},{g17(b)},{g17(c)},{g17(d)}")
    hx = (db.row_lx + db.row_step * db.row_num_sites.astype(f32)).astype(f32)
    hy = (db.row_ly + db.row_height).astype(f32)
    for r in range(db.row_ly.size):
        lines.append(f"row,{r},{g17(db.row_lx[r])},{g17(db.row_ly[r])},{g17(hx[r])},{g17(hy[r])}")
    with open(os.path.join(out_dir, "geometry.csv"), "w") as f:
        f.write("\n".join(lines) + "\n")


def _probes(ev, db, params, x, y, idx, g, dens, comb):
    """The six probes (diagnostics.cpp:154-172): the opt nodes moved by 1%, 10% and 100% of a bin
    along the density direction and along the combined direction (the largest node move scaled
    to that), clamped into the core, and the overflow and energy of a fresh grid there."""
    n = idx.size
    w, h = db.node_w[idx], db.node_h[idx]
    half, eps = f32(0.5), f32(1e-3)
    clx, cly, chx, chy = (f32(v) for v in db.core)
    xlo = (clx + half * w + eps).astype(f32)
    ylo = (cly + half * h + eps).astype(f32)
    xhi = np.maximum(xlo, (chx - half * w - eps).astype(f32))
    yhi = np.maximum(ylo, (chy - half * h - eps).astype(f32))
    step = float(min(f32(g["step_x"]), f32(g["step_y"])))
    out = []
    for direction, v in (("density", dens), ("combined", comb)):
        norm = float(np.max(np.hypot(v[:n].astype(np.float64), v[n:].astype(np.float64)))) if n else 0.0
        for fraction in (0.01, 0.1, 1.0):
            scale = fraction * step / norm if norm > 0 else 0.0
            tx, ty = x.copy(), y.copy()
            mx = (x[idx] + (scale * v[:n].astype(np.float64)).astype(f32)).astype(f32)
            my = (y[idx] + (scale * v[n:].astype(np.float64)).astype(f32)).astype(f32)
            tx[idx] = np.minimum(np.maximum(mx, xlo), xhi)
            ty[idx] = np.minimum(np.maximum(my, ylo), yhi)
            e = ev.at(tx, ty)
            out.append({"direction": direction, "fraction_of_bin": fraction, "overflow": float(f32(e["overflow"])),
                        "energy": _energy(e["maps"])})
    return out
