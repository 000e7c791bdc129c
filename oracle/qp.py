"""CPU restatement of the reference's B2B (Kraftwerk2) quadratic initial placement, in numpy.
Test infrastructure only: the tests use it as the checker for superplace_b200.qp.

- bound_pins        computeNetBoundPins      src/db/hpwl.cpp:70-103
- b2b_pairs         forEachB2BPair           src/init/b2b_model.h:57-82
- assemble          assemble<A>              src/init/quadratic_placer.cpp:43-112, with Eigen
                    3.4.0's SparseMatrix::setFromTriplets (equal (row, col) triplets summed in
                    emission order after the seeded zero diagonal)
- bicgstab          Eigen 3.4.0 BiCGSTAB with DiagonalPreconditioner (van der Vorst 1992;
                    restart when |r0.r| < eps^2 |r0|^2), in float32 with numpy's dot products
- place             QuadraticPlacer::place   src/init/quadratic_placer.cpp:153-228

Eigen is not shipped with the reference and is not installed here, so the reference's solver
cannot be run: the pair rule is pinned by the identity of test/test_b2b.cpp, the assembly is
exact float32 arithmetic in the reference's order, and the solver is checked by tolerance.
Pure-Python loops: small designs only.
"""
from __future__ import annotations

import numpy as np

f32 = np.float32


def pin_pos(db, pos, off, p):
    return f32(pos[db.pin2node[p]]) + f32(off[p])


def bound_pins(db, x, y):
    nets = db.num_nets
    out = [np.full(nets, -1, np.int64) for _ in range(4)]
    for k in range(nets):
        b, e = int(db.net2pin_start[k]), int(db.net2pin_start[k + 1])
        if b == e:
            continue
        p0 = int(db.flat_net2pin[b])
        idx = [p0, p0, p0, p0]
        xl = xh = pin_pos(db, x, db.pin_offset_x, p0)
        yl = yh = pin_pos(db, y, db.pin_offset_y, p0)
        for t in range(b + 1, e):
            p = int(db.flat_net2pin[t])
            px, py = pin_pos(db, x, db.pin_offset_x, p), pin_pos(db, y, db.pin_offset_y, p)
            if px < xl:
                xl, idx[0] = px, p
            if px > xh:
                xh, idx[1] = px, p
            if py < yl:
                yl, idx[2] = py, p
            if py > yh:
                yh, idx[3] = py, p
        for a in range(4):
            out[a][k] = idx[a]
    return out  # x lo, x hi, y lo, y hi


def b2b_pairs(db, k, lo, hi, pos, off, weight, min_distance, drop_lower_bound_of_p=False):
    """(p, q, w) of net k in the reference's (s, t) order. `drop_lower_bound_of_p` plants the
    mistake test/test_b2b.cpp:159-196 guards against (the p == lo test left out)."""
    b, e = int(db.net2pin_start[k]), int(db.net2pin_start[k + 1])
    deg = e - b
    if deg < 2:
        return []
    coef = f32(f32(1.0 if weight is None else weight[k]) / f32(deg - 1))
    min_d = max(f32(1e-6), f32(min_distance))
    out = []
    for s in range(b, e):
        p = int(db.flat_net2pin[s])
        for t in range(s + 1, e):
            q = int(db.flat_net2pin[t])
            if db.pin2node[p] == db.pin2node[q]:
                continue
            p_bound = (p == hi) if drop_lower_bound_of_p else (p == lo or p == hi)
            if not p_bound and not (q == lo or q == hi):
                continue
            d = abs(f32(pin_pos(db, pos, off, p) - pin_pos(db, pos, off, q)))
            out.append((p, q, f32(coef / max(d, min_d))))
    return out


def assemble(db, axis, x, y, weight=None, min_distance=1.0, ignore_net_degree=100):
    """(row_start, col, val, rhs) of one axis, float32 sums in the reference's order."""
    n = db.num_movable
    pos = x if axis == 0 else y
    off = db.pin_offset_x if axis == 0 else db.pin_offset_y
    lo_all, hi_all = bound_pins(db, x, y)[2 * axis: 2 * axis + 2]
    entries = {(i, i): f32(0.0) for i in range(n)}
    rhs = [f32(0.0)] * n
    min_d = max(f32(1e-6), f32(min_distance))

    def add(i, j, v):
        entries[(i, j)] = f32(entries.get((i, j), None) + v) if (i, j) in entries else f32(v)

    for k in range(db.num_nets):
        deg = int(db.net2pin_start[k + 1] - db.net2pin_start[k])
        if deg < 2 or deg > ignore_net_degree:
            continue
        for p, q, w in b2b_pairs(db, k, int(lo_all[k]), int(hi_all[k]), pos, off, weight, min_d):
            ni, nj = int(db.pin2node[p]), int(db.pin2node[q])
            oi, oj = f32(off[p]), f32(off[q])
            mi, mj = ni < n, nj < n
            if mi and mj:
                add(ni, ni, w)
                add(nj, nj, w)
                add(ni, nj, -w)
                add(nj, ni, -w)
                rhs[ni] = f32(rhs[ni] + f32(-w * f32(oi - oj)))
                rhs[nj] = f32(rhs[nj] + f32(-w * f32(oj - oi)))
            elif mi:
                add(ni, ni, w)
                rhs[ni] = f32(rhs[ni] + f32(w * f32(pin_pos(db, pos, off, q) - oi)))
            elif mj:
                add(nj, nj, w)
                rhs[nj] = f32(rhs[nj] + f32(w * f32(pin_pos(db, pos, off, p) - oj)))
    for i in range(n):
        if entries[(i, i)] == 0:
            entries[(i, i)] = f32(1e-6)
            rhs[i] = f32(rhs[i] + f32(f32(1e-6) * f32(pos[i])))
    keys = sorted(entries)
    start = np.zeros(n + 1, np.int32)
    for i, _ in keys:
        start[i + 1] += 1
    start = np.cumsum(start).astype(np.int32)
    col = np.array([j for _, j in keys], np.int32)
    val = np.array([entries[kk] for kk in keys], np.float32)
    return start, col, val, np.array(rhs, np.float32)


def spmv(start, col, val, v):
    out = np.zeros(start.shape[0] - 1, np.float32)
    prod = (val * v[col]).astype(np.float32)
    np.add.at(out, np.repeat(np.arange(out.shape[0]), np.diff(start)), prod)
    return out


def bicgstab(start, col, val, b, x, max_iter, tol):
    """Returns (x, iterations, error)."""
    n = b.shape[0]
    diag = np.ones(n, np.float32)
    for i in range(n):
        for k in range(start[i], start[i + 1]):
            if col[k] == i and val[k] != 0:
                diag[i] = f32(1.0) / val[k]
    x = x.astype(np.float32).copy()
    dot = lambda u, v: f32(np.dot(u, v))  # noqa: E731
    r = (b - spmv(start, col, val, x)).astype(np.float32)
    r0 = r.copy()
    r0_sq = dot(r0, r0)
    b_sq = dot(b, b)
    if b_sq == 0:
        return np.zeros(n, np.float32), max_iter, f32(tol)
    rho = alpha = w = f32(1.0)
    v = np.zeros(n, np.float32)
    p = np.zeros(n, np.float32)
    tol2 = f32(f32(tol) * f32(tol) * b_sq)
    eps2 = f32(np.finfo(np.float32).eps) ** 2
    it = restarts = 0
    while dot(r, r) > tol2 and it < max_iter:
        rho_old = rho
        rho = dot(r0, r)
        if abs(rho) < eps2 * r0_sq:
            r = (b - spmv(start, col, val, x)).astype(np.float32)
            r0 = r.copy()
            rho = r0_sq = dot(r, r)
            if restarts == 0:
                it = 0
            restarts += 1
        beta = f32(f32(rho / rho_old) * f32(alpha / w))
        p = (r + beta * (p - w * v)).astype(np.float32)
        y = (diag * p).astype(np.float32)
        v = spmv(start, col, val, y)
        alpha = f32(rho / dot(r0, v))
        s = (r - alpha * v).astype(np.float32)
        z = (diag * s).astype(np.float32)
        t = spmv(start, col, val, z)
        tt = dot(t, t)
        w = f32(dot(t, s) / tt) if tt > 0 else f32(0.0)
        x = (x + (alpha * y + w * z)).astype(np.float32)
        r = (s - w * t).astype(np.float32)
        it += 1
    return x, it, f32(np.sqrt(dot(r, r) / b_sq))


def hpwl(db, x, y):
    total = 0.0
    for k in range(db.num_nets):
        b, e = int(db.net2pin_start[k]), int(db.net2pin_start[k + 1])
        if e - b < 2:
            continue
        pins = db.flat_net2pin[b:e]
        px = (x[db.pin2node[pins]] + db.pin_offset_x[pins]).astype(np.float32)
        py = (y[db.pin2node[pins]] + db.pin_offset_y[pins]).astype(np.float32)
        total += float(f32(px.max() - px.min())) + float(f32(py.max() - py.min()))
    return total


def place(db, weight=None, max_iter=20, tol=1e-6, solver_max_iter=100, outer_tol=1e-4, min_distance=1.0,
          ignore_net_degree=100):
    """Positions after QuadraticPlacer::place and its per-iteration HPWL."""
    n = db.num_movable
    x = db.node_x.astype(np.float32).copy()
    y = db.node_y.astype(np.float32).copy()
    if n == 0:
        return x, y, []
    x[:n] = f32(f32(0.5) * f32(f32(db.core[0]) + f32(db.core[2])))
    y[:n] = f32(f32(0.5) * f32(f32(db.core[1]) + f32(db.core[3])))
    sol = [x[:n].copy(), y[:n].copy()]
    hist = []
    last = 0.0
    it = 0
    while True:
        for axis in (0, 1):
            pos = x if axis == 0 else y
            start, col, val, rhs = assemble(db, axis, x, y, weight, min_distance, ignore_net_degree)
            s, _, _ = bicgstab(start, col, val, rhs, sol[axis], solver_max_iter, tol)
            size = db.node_w if axis == 0 else db.node_h
            lo_c, hi_c = (db.core[0], db.core[2]) if axis == 0 else (db.core[1], db.core[3])
            for i in range(n):
                v = s[i] if np.isfinite(s[i]) else pos[i]
                half = f32(f32(0.5) * f32(size[i]))
                lo, hi = f32(f32(lo_c) + half), f32(f32(hi_c) - half)
                v = min(max(f32(v), lo), hi) if lo <= hi else f32(f32(0.5) * f32(lo + hi))
                pos[i] = v
                s[i] = v
            sol[axis] = s
        h = hpwl(db, x, y)
        hist.append(h)
        stalled = it > 4 and last > 0 and abs(h - last) < outer_tol * last
        last = h
        if stalled or it + 1 >= max_iter:
            break
        it += 1
    return x, y, hist
