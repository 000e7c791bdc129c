"""Seeded synthetic netlists for the placement workloads.

No public benchmark suite is available here; these generators produce instances with the
shapes, sizes and value distributions of the measured configurations:

* ``small_design``  (2,000 cells, 600x600 die, 64 IO pads, 2,100 nets, 64x64 bins)
* ``large_design``  (211k cells, 11,600x11,600 die, 543 fixed macros covering 35%,
                     221k nets, 512x512 bins)
* ``mixed_design``  (``large_design`` + 63 movable macros at 56.9% of movable area,
                     fixed macros cut to 200, 1024x1024 bins)
* ``served_design`` (the small generator rescaled: 1k-100k cells, grid 64..512)

Nets: degree 2 (60%), 3 (18%), 4-5 (12%), 6-20 (9%), 21-64 (1%); each net draws distinct
cells from a window of +-50 positions around a random anchor in a random cell ordering
(local connectivity), pin offsets uniform inside the cell. Pins are stored net by net,
so flat_net2pin is the identity, as in a BookShelf .nets file.

Initial placement: the reference starts mGP from a quadratic (B2B) placement, which is
outside this path. These instances start from a seeded Gaussian cluster around the core
centre (sigma = core/20), the same "cells piled near the centre" situation the reference's
own GP regression fixture uses (test/test_eplace.cpp:45-56).
"""
from __future__ import annotations

import numpy as np

from .placedb import F_FIXED, F_MACRO, PlaceDB

DEGREE_BINS = ((2, 2, 0.60), (3, 3, 0.18), (4, 5, 0.12), (6, 20, 0.09), (21, 64, 0.01))


def _degrees(rng, n_nets):
    probs = np.array([b[2] for b in DEGREE_BINS])
    which = rng.choice(len(DEGREE_BINS), size=n_nets, p=probs / probs.sum())
    lo = np.array([b[0] for b in DEGREE_BINS])[which]
    hi = np.array([b[1] for b in DEGREE_BINS])[which]
    return (lo + np.floor(rng.random(n_nets) * (hi - lo + 1))).astype(np.int64)


def _local_nets(rng, n_cells, n_nets, window=50):
    """Pin node lists (flat) and net ids for local-connectivity nets over cells 0..n-1."""
    order = rng.permutation(n_cells)
    deg = _degrees(rng, n_nets)
    span = 2 * window + 1
    if n_cells < span:
        span = n_cells
    deg = np.minimum(deg, span)
    anchor = rng.integers(0, n_cells, n_nets)
    start = np.clip(anchor - window, 0, max(n_cells - span, 0))
    pin_node = np.empty(int(deg.sum()), np.int64)
    net_of_pin = np.repeat(np.arange(n_nets), deg)
    offs = np.concatenate([[0], np.cumsum(deg)])
    for d in np.unique(deg):
        idx = np.nonzero(deg == d)[0]
        for c0 in range(0, idx.size, 1 << 16):
            sel = idx[c0:c0 + (1 << 16)]
            keys = rng.random((sel.size, span), dtype=np.float32)
            pick = np.argpartition(keys, d - 1, axis=1)[:, :d] if d < span else \
                np.tile(np.arange(span), (sel.size, 1))
            pick = np.sort(pick, axis=1)
            cells = order[start[sel, None] + pick]
            dst = offs[sel, None] + np.arange(d)[None, :]
            pin_node[dst.ravel()] = cells.ravel()
    return pin_node, net_of_pin, deg


def _rows(n_rows, row_h, width, ly0=0.0):
    ly = (ly0 + row_h * np.arange(n_rows)).astype(np.float32)
    return (ly, np.full(n_rows, row_h, np.float32), np.zeros(n_rows, np.float32),
            np.ones(n_rows, np.float32), np.full(n_rows, int(width), np.int32))


def _cluster_xy(rng, n, core, w, h, sigma_frac=0.05):
    lx, ly, hx, hy = core
    cx, cy = 0.5 * (lx + hx), 0.5 * (ly + hy)
    x = cx + rng.normal(0.0, sigma_frac * (hx - lx), n)
    y = cy + rng.normal(0.0, sigma_frac * (hy - ly), n)
    x = np.clip(x, lx + 0.5 * w, hx - 0.5 * w)
    y = np.clip(y, ly + 0.5 * h, hy - 0.5 * h)
    return x.astype(np.float32), y.astype(np.float32)


def _place_macros(rng, ws, hs, core, max_tries=4000):
    """Non-overlapping random placement of fixed macros, largest first (rejection)."""
    lx, ly, hx, hy = core
    order = np.argsort(-(ws * hs))
    xs = np.zeros_like(ws)
    ys = np.zeros_like(hs)
    placed = []
    boxes = np.zeros((0, 4))
    for i in order:
        w, h = ws[i], hs[i]
        ok = False
        for _ in range(max_tries):
            x = rng.uniform(lx + 0.5 * w, hx - 0.5 * w)
            y = rng.uniform(ly + 0.5 * h, hy - 0.5 * h)
            b = np.array([x - 0.5 * w, y - 0.5 * h, x + 0.5 * w, y + 0.5 * h])
            if boxes.shape[0] == 0 or not np.any(
                    (boxes[:, 0] < b[2]) & (b[0] < boxes[:, 2]) &
                    (boxes[:, 1] < b[3]) & (b[1] < boxes[:, 3])):
                ok = True
                break
        if not ok:  # give up on non-overlap for this one (rare)
            x = rng.uniform(lx + 0.5 * w, hx - 0.5 * w)
            y = rng.uniform(ly + 0.5 * h, hy - 0.5 * h)
            b = np.array([x - 0.5 * w, y - 0.5 * h, x + 0.5 * w, y + 0.5 * h])
        xs[i], ys[i] = x, y
        boxes = np.vstack([boxes, b])
        placed.append(i)
    return xs.astype(np.float32), ys.astype(np.float32)


def build_design(*, seed, die, row_h, n_cells, cell_w, n_nets, n_fixed_macros=0,
                 fixed_cover=0.0, macro_rows=(20, 400), n_movable_macros=0,
                 movable_macro_frac=0.0, movable_macro_rows=(40, 300), n_pads=0,
                 pad_size=4.0, name="design") -> PlaceDB:
    rng = np.random.default_rng(seed)
    n_rows = int(die // row_h)
    rows = _rows(n_rows, row_h, die)
    core = (0.0, 0.0, float(die), float(n_rows * row_h))

    cell_w = np.asarray(cell_w, np.float32)
    cell_h = np.full(n_cells, row_h, np.float32)
    cell_area = float(np.sum(cell_w.astype(np.float64) * row_h))

    # movable macros (mixed-size designs)
    mm_w = np.zeros(0, np.float32)
    mm_h = np.zeros(0, np.float32)
    if n_movable_macros:
        hr = np.exp(rng.normal(np.log(90.0), 0.6, n_movable_macros))
        hr = np.clip(hr, *movable_macro_rows)
        mh = (np.round(hr) * row_h).astype(np.float64)
        aspect = np.exp(rng.normal(0.0, 0.3, n_movable_macros))
        mw = mh * aspect
        target = movable_macro_frac / (1.0 - movable_macro_frac) * cell_area
        s = np.sqrt(target / np.sum(mw * mh))
        mw = np.maximum(np.round(mw * s), 8.0)
        mh = np.clip(np.round(mh * s / row_h), movable_macro_rows[0], movable_macro_rows[1]) * row_h
        mm_w, mm_h = mw.astype(np.float32), mh.astype(np.float32)

    # fixed macros
    fm_w = np.zeros(0, np.float32)
    fm_h = np.zeros(0, np.float32)
    if n_fixed_macros:
        hr = np.clip(np.exp(rng.normal(np.log(40.0), 0.5, n_fixed_macros)), *macro_rows)
        h = hr * row_h
        aspect = np.exp(rng.normal(0.0, 0.4, n_fixed_macros))
        w = h * aspect
        target = fixed_cover * die * die
        s = np.sqrt(target / np.sum(w * h))
        w, h = np.round(w * s), np.round(h * s)
        fm_w = np.clip(w, 8, 0.25 * die).astype(np.float32)
        fm_h = np.clip(h, row_h, 0.25 * die).astype(np.float32)

    n_mm, n_fm = mm_w.size, fm_w.size
    n_mov = n_cells + n_mm
    db = PlaceDB()
    db.name = name
    node_w = np.concatenate([cell_w, mm_w, fm_w, np.full(n_pads, pad_size, np.float32)])
    node_h = np.concatenate([cell_h, mm_h, fm_h, np.full(n_pads, pad_size, np.float32)])
    flags = np.concatenate([np.zeros(n_cells, np.uint8), np.full(n_mm, F_MACRO, np.uint8),
                            np.full(n_fm, F_FIXED, np.uint8), np.full(n_pads, F_FIXED, np.uint8)])
    cx, cy = _cluster_xy(rng, n_mov, core, node_w[:n_mov], node_h[:n_mov])
    fx, fy = _place_macros(rng, fm_w.astype(np.float64), fm_h.astype(np.float64), core) \
        if n_fm else (np.zeros(0, np.float32), np.zeros(0, np.float32))
    # IO pads: evenly spaced around the core boundary, centred on it
    if n_pads:
        per = n_pads // 4
        t = (np.arange(per) + 0.5) / per
        W, H = core[2], core[3]
        px = np.concatenate([t * W, np.full(per, W), (1 - t) * W, np.zeros(per)])
        py = np.concatenate([np.zeros(per), t * H, np.full(per, H), (1 - t) * H])
        extra = n_pads - 4 * per
        px = np.concatenate([px, np.zeros(extra)])
        py = np.concatenate([py, np.zeros(extra)])
    else:
        px = py = np.zeros(0)
    db.node_x = np.concatenate([cx, fx, px.astype(np.float32)]).astype(np.float32)
    db.node_y = np.concatenate([cy, fy, py.astype(np.float32)]).astype(np.float32)
    db.node_w, db.node_h, db.node_flags = node_w, node_h, flags
    db.num_movable = n_mov
    db.num_nodes = n_mov + n_fm + n_pads

    # nets over the movable nodes (cells and movable macros share the ordering)
    pin_node, net_of_pin, _ = _local_nets(rng, n_mov, n_nets)
    # every fixed macro and pad joins a few nets (anchors the netlist to the die)
    extra_nodes = np.arange(n_mov, db.num_nodes)
    if extra_nodes.size:
        k = np.where(extra_nodes < n_mov + n_fm, 4, 1)
        en = np.repeat(extra_nodes, k)
        enet = rng.integers(0, n_nets, en.size)
        pin_node = np.concatenate([pin_node, en])
        net_of_pin = np.concatenate([net_of_pin, enet])
    order = np.argsort(net_of_pin, kind="stable")
    pin_node, net_of_pin = pin_node[order], net_of_pin[order]
    w_p = node_w[pin_node].astype(np.float64)
    h_p = node_h[pin_node].astype(np.float64)
    db.pin_offset_x = ((rng.random(pin_node.size) - 0.5) * w_p).astype(np.float32)
    db.pin_offset_y = ((rng.random(pin_node.size) - 0.5) * h_p).astype(np.float32)
    db.pin2node = pin_node.astype(np.int32)
    db.finalize_csr(net_of_pin.astype(np.int32), n_nets)
    db.row_ly, db.row_height, db.row_lx, db.row_step, db.row_num_sites = rows
    db.compute_regions()
    db.extend_node2pin()
    return db


def small_design(seed=1002) -> PlaceDB:
    """600x600 die, 50 rows of 12, 2,000 cells (w in 2..16), 64 pads, 2,100 nets."""
    rng = np.random.default_rng(seed + 17)
    w = rng.integers(2, 17, 2000).astype(np.float32)
    return build_design(seed=seed, die=600.0, row_h=12.0, n_cells=2000, cell_w=w,
                        n_nets=2100, n_pads=64, name="small_2k")


def large_design(seed=1002, n_cells=211_000, n_nets=221_000) -> PlaceDB:
    """11,600 die, 211k cells (log-normal widths, median 6, 1..40), 543 fixed macros at 35%."""
    rng = np.random.default_rng(seed + 17)
    w = np.clip(np.round(np.exp(rng.normal(np.log(6.0), 0.55, n_cells))), 1, 40)
    return build_design(seed=seed, die=11600.0, row_h=12.0, n_cells=n_cells,
                        cell_w=w.astype(np.float32), n_nets=n_nets, n_fixed_macros=543,
                        fixed_cover=0.35, name="large_211k")


def mixed_design(seed=1002, n_cells=211_000, n_nets=None) -> PlaceDB:
    """large_design + 63 movable macros (56.9% of movable area), 200 fixed macros. Fewer cells
    shrink the die with the square root of the count (same utilisation); nets default to
    1.047 x cells (221k at 211k)."""
    rng = np.random.default_rng(seed + 17)
    w = np.clip(np.round(np.exp(rng.normal(np.log(6.0), 0.55, n_cells))), 1, 40)
    n_nets = int(round(n_cells * 221_000 / 211_000)) if n_nets is None else n_nets
    die = 11600.0 if n_cells == 211_000 else float(np.ceil(11600.0 * np.sqrt(n_cells / 211_000) / 12.0) * 12.0)
    return build_design(seed=seed, die=die, row_h=12.0, n_cells=n_cells,
                        cell_w=w.astype(np.float32), n_nets=n_nets, n_fixed_macros=200,
                        fixed_cover=0.12, n_movable_macros=63, movable_macro_frac=0.569,
                        name="mixed_211k")


def scaled_design(seed, n_cells) -> tuple[PlaceDB, int]:
    """Serving request: the small generator at n_cells, ~60% utilisation, nets = 1.05x
    cells, grid = next power of two in 64..512 at ~4 cells per bin. Returns (db, grid)."""
    rng = np.random.default_rng(seed + 17)
    w = rng.integers(2, 17, n_cells).astype(np.float32)
    area = float(np.sum(w)) * 12.0 / 0.6
    die = float(np.ceil(np.sqrt(area) / 12.0) * 12.0)
    g = 64
    while g < 512 and g * g * 4 < n_cells:
        g *= 2
    db = build_design(seed=seed, die=die, row_h=12.0, n_cells=n_cells, cell_w=w,
                      n_nets=int(round(1.05 * n_cells)), n_pads=64, name=f"served_{n_cells}")
    return db, g
