"""Solver-agnostic restatements of the reference's known-answer tests for the GP path, so
the same checks run against the oracle (CPU) and against the CUDA path (GPU):

* poisson_analytic   — test/test_poisson.cpp:80-262 (six analytic checks)
* density_semantics  — test/test_density.cpp:60-246
* wa_central_diff    — test/test_wirelength.cpp:19-185
"""
from __future__ import annotations

import numpy as np

from superplace_b200.placedb import F_FILLER, F_FIXED, F_MACRO, make_db

KN, KSTEP = 64, 2.5  # test_poisson.cpp:31-32


def _remove_dc(v):
    return (v - np.float32(v.astype(np.float64).mean())).astype(np.float32)


def _gaussian(n, cx, cy, sigma, amp=1.0):
    x = (np.arange(n, dtype=np.float32) + 0.5)[:, None] - np.float32(cx)
    y = (np.arange(n, dtype=np.float32) + 0.5)[None, :] - np.float32(cy)
    return (amp * np.exp(-(x * x + y * y) / (2.0 * sigma * sigma))).astype(np.float32)


def poisson_analytic(solve, tol_scale=1.0, n=KN):
    """solve(rho[n][n], step) -> (phi, xi_x, xi_y). Asserts the six checks (the reference
    runs them at n = 64; tensor-core tiles need n >= 128)."""
    st = KSTEP
    c = 0.5 * n
    # 1: Gaussian field points outward, boundary normal small (test_poisson.cpp:81-127)
    rho = _remove_dc(_gaussian(n, c, c, n / 10.0))
    assert abs(rho.astype(np.float64).mean()) < 1e-6
    phi, ex, ey = solve(rho, st)
    scale = np.abs(ex).max() + np.abs(ey).max()
    xs = np.arange(n) + 0.5 - c
    dx, dy = np.meshgrid(xs, xs, indexing="ij")
    r = np.sqrt(dx * dx + dy * dy)
    sel = (r >= 3.0) & (r <= 0.4 * n) & (np.sqrt(ex * ex + ey * ey) >= 1e-3 * scale)
    assert sel.sum() > 100
    assert (dx * ex + dy * ey > 0)[sel].sum() >= int(0.99 * sel.sum())
    normal = max(np.abs(ex[0]).max(), np.abs(ex[-1]).max(), np.abs(ey[:, 0]).max(), np.abs(ey[:, -1]).max())
    assert normal < 0.05 * scale
    # 2: uniform density -> zero field (test_poisson.cpp:130-140)
    phi, ex, ey = solve(_remove_dc(np.full((n, n), 3.7, np.float32)), st)
    assert np.abs(ex).max() < 1e-4 and np.abs(ey).max() < 1e-4
    # 3: mirror symmetry -> antisymmetric field (test_poisson.cpp:143-167)
    x = np.arange(n, dtype=np.float32) + 0.5 - 0.5 * n
    yv = np.arange(n, dtype=np.float32)
    rho = (np.exp(-x * x / 50.0)[:, None] * (1.0 + 0.3 * np.sin(0.2 * yv))[None, :]).astype(np.float32)
    phi, ex, ey = solve(_remove_dc(rho), st)
    assert np.abs(ex + ex[::-1]).max() < 1e-3 * np.abs(ex).max() * tol_scale
    # 4: single mode phi/rho = 1/(u^2+v^2) (test_poisson.cpp:173-201)
    j0, k0 = 3, 5
    u = np.float32(np.pi * j0 / (n * st))
    v = np.float32(np.pi * k0 / (n * st))
    xx = np.arange(n, dtype=np.float32) + 0.5
    rho = (np.cos(np.float32(np.pi) * j0 * xx / n)[:, None] *
           np.cos(np.float32(np.pi) * k0 * xx / n)[None, :]).astype(np.float32)
    phi, ex, ey = solve(rho, st)
    expect = 1.0 / (u * u + v * v)
    m = np.abs(rho) >= 0.1
    assert (np.abs(phi[m] / rho[m] - expect) / expect).max() < 1e-4 * tol_scale
    # 5: xi = -grad phi by central differences (test_poisson.cpp:207-237)
    rho = (np.cos(np.float32(np.pi) * 2 * xx / n)[:, None] * np.cos(np.float32(np.pi) * 3 * xx / n)[None, :] +
           0.5 * np.cos(np.float32(np.pi) * xx / n)[:, None]).astype(np.float32)
    phi, ex, ey = solve(_remove_dc(rho), st)
    gx = (phi[2:, 1:-1] - phi[:-2, 1:-1]) / (2.0 * st)
    gy = (phi[1:-1, 2:] - phi[1:-1, :-2]) / (2.0 * st)
    assert np.abs(ex[1:-1, 1:-1] + gx).max() < 0.01 * np.abs(ex).max()
    assert np.abs(ey[1:-1, 1:-1] + gy).max() < 0.01 * np.abs(ey).max()
    # 6: determinism (test_poisson.cpp:240-262)
    rho = _remove_dc(_gaussian(n, 0.3 * n, 0.7 * n, 5.0))
    a = solve(rho, st)
    b = solve(rho.copy(), st)
    for p, q in zip(a, b):
        assert np.array_equal(p, q)


def _db(size, cells):
    return make_db(cells, [(0.0, size, 0.0, 1.0, int(size))])


def density_semantics(make_grid):
    """make_grid(db, target, dim) -> object with accumulate() -> (node, filler) maps,
    overflow() -> tau, total_charge(). Asserts test_density.cpp's criteria."""
    # scaling rule (test_density.cpp:62-83)
    gc = make_grid(_db(64.0, [(32, 32, 16, 16, 0)]), 0.5, 8)
    gm = make_grid(_db(64.0, [(32, 32, 16, 16, F_MACRO)]), 0.5, 8)
    sc = gc.accumulate()[0].astype(np.float64).sum()
    sm = gm.accumulate()[0].astype(np.float64).sum()
    assert abs(sc - 256.0) < 1e-3 and abs(sm - 128.0) < 1e-3
    # filler separate (test_density.cpp:86-95)
    g = make_grid(_db(64.0, [(32, 32, 16, 16, F_FILLER)]), 0.5, 8)
    nd, fd = g.accumulate()
    assert abs(nd.astype(np.float64).sum()) < 1e-4 and abs(fd.astype(np.float64).sum() - 256.0) < 1e-3
    # local smoothing conserves area (test_density.cpp:99-116)
    g = make_grid(_db(64.0, [(32, 32, 2, 2, 0)]), 1.0, 8)
    nd, _ = g.accumulate()
    assert abs(nd.astype(np.float64).sum() - 4.0) < 1e-3
    assert (nd > 1e-6).sum() > 1
    # tau = 0 when exactly balanced (test_density.cpp:120-136)
    cells = [(4 + 8 * i, 4 + 8 * j, 8, 8, 0) for i in range(8) for j in range(8)]
    g = make_grid(_db(64.0, cells), 1.0, 8)
    g.accumulate()
    assert abs(g.overflow()) < 1e-4
    # tau > 0.5 when stacked (test_density.cpp:139-151)
    g = make_grid(_db(64.0, [(4, 4, 8, 8, 0)] * 64), 1.0, 8)
    g.accumulate()
    assert g.overflow() > 0.5
    # tau excludes fillers (test_density.cpp:154-173)
    base = [(4, 4, 8, 8, 0)] * 32
    ga = make_grid(_db(64.0, base), 1.0, 8)
    gb = make_grid(_db(64.0, base + [(4, 4, 8, 8, F_FILLER)] * 32), 1.0, 8)
    ga.accumulate()
    gb.accumulate()
    assert abs(ga.overflow() - gb.overflow()) < 1e-5
    # total charge == total density (test_density.cpp:183-205)
    cells = ([(20 + 4 * i, 30, 6, 6, 0) for i in range(20)] +
             [(30 + 18 * i, 70, 16, 16, F_MACRO) for i in range(5)] +
             [(25 + 7 * i, 100, 5, 5, F_FILLER) for i in range(12)])
    g = make_grid(_db(128.0, cells), 0.6, 16)
    nd, fd = g.accumulate()
    dens = nd.astype(np.float64).sum() + fd.astype(np.float64).sum()
    assert abs(g.total_charge() - dens) <= 1e-3 * max(dens, 1.0)
    # determinism (test_density.cpp:209-232)
    cells = [(10 + (i * 37) % 236, 10 + (i * 61) % 236, 6, 6, 0) for i in range(2000)]
    db = _db(256.0, cells)
    a = make_grid(db, 1.0, 32).accumulate()
    b = make_grid(db, 1.0, 32).accumulate()
    assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])


def wirelength_db(n_mov, n_fixed, nets, seed):
    """test_wirelength.cpp:19-57 fixture: movable 6x12 nodes, fixed 20x20, positions in
    [100, 900), pin offsets in [-4, 4) (seeded; the reference's mt19937 stream is not
    reproduced, the fixture shape is)."""
    rng = np.random.default_rng(seed)
    nodes = [(0, 0, 6, 12, 0)] * n_mov + [(0, 0, 20, 20, F_FIXED)] * n_fixed
    pos = rng.uniform(100, 900, (n_mov + n_fixed, 2))
    nodes = [(pos[i, 0], pos[i, 1], nd[2], nd[3], nd[4]) for i, nd in enumerate(nodes)]
    npins = sum(len(n) for n in nets)
    offs = rng.uniform(-4, 4, (npins, 2))
    return make_db(nodes, [(0.0, 1000.0, 0.0, 1.0, 1000)], nets, offs)


WA_CASES = [
    ("3-pin", (3, 0, [[0, 1, 2]], 11), [50.0]),
    ("fixed pin", (3, 1, [[0, 1, 2, 3]], 22), [50.0]),
    ("shared", (5, 0, [[0, 1, 2], [1, 3], [2, 3, 4], [0, 4]], 33), [50.0]),
    ("gamma sweep", (6, 2, [[0, 1, 2, 6], [2, 3, 4], [4, 5, 7], [0, 5]], 44), [500.0, 50.0, 5.0]),
    ("40-pin", (40, 0, [list(range(40))], 55), [20.0]),
]


def wa_central_diff(wa_fn):
    """wa_fn(db, gamma) -> (wl, grad[2*numMovable]); central differences with h = 0.5,
    error / max|grad| < 1e-3 (test_wirelength.cpp:67-112)."""
    for _, args, gammas in WA_CASES:
        db = wirelength_db(*args)
        n = db.num_movable
        for gamma in gammas:
            _, grad = wa_fn(db, gamma)
            denom = max(np.abs(grad).max(), 1e-9)
            worst = 0.0
            for i in range(n):
                for axis in range(2):
                    arr = db.node_x if axis == 0 else db.node_y
                    saved = arr[i]
                    arr[i] = saved + np.float32(0.5)
                    wp, _ = wa_fn(db, gamma)
                    arr[i] = saved - np.float32(0.5)
                    wm, _ = wa_fn(db, gamma)
                    arr[i] = saved
                    num = (wp - wm) / 1.0
                    worst = max(worst, abs(num - grad[axis * n + i]) / denom)
            assert worst < 1e-3, (args, gamma, worst)
    # tiny gamma stays finite (test_wirelength.cpp:140-153)
    db = wirelength_db(8, 0, [[0, 1, 2, 3], [4, 5, 6, 7]], 66)
    wl, grad = wa_fn(db, 0.01)
    assert np.isfinite(wl) and np.all(np.isfinite(grad))
    # WA rises towards HPWL as gamma shrinks (test_wirelength.cpp:156-172)
    db = wirelength_db(10, 0, [[0, 1, 2, 3, 4], [5, 6, 7, 8, 9], [0, 9]], 77)
    prev = -1.0
    for gamma in (200.0, 50.0, 10.0, 1.0):
        wl, _ = wa_fn(db, gamma)
        if prev >= 0:
            assert wl >= prev - 1e-3
        prev = wl


# ---- the reference's host legalisers (oracle/_ref), as the callables superplace_b200.flow takes
def _to_ref(db):
    from oracle import ref

    return ref.RefDb(db)


def _back(db, r):
    x, y, _, _, flags = r.nodes()
    n = db.total_nodes
    db.node_x[:n], db.node_y[:n] = x[:n], y[:n]
    db.node_flags[:n] = flags[:n]


def ref_legalize_cells(db) -> dict:
    """The reference's LegalizeStage body: legalizeCells (src/lg/abacus.cpp:155-284) on db."""
    from oracle import ref

    r = _to_ref(db)
    res = ref.abacus(r)
    _back(db, r)
    return res


def ref_legalize_macros(params):
    """The reference's legalizeMacros (src/lg/macro_sa.cpp:493) as a flow.global_place mLG
    callable; it leaves every macro F_FIXED."""

    def run(db) -> dict:
        r = _to_ref(db)
        res = r.legalize_macros(params)
        _back(db, r)
        return res

    return run


def overfull_design(seed=7):
    """A design that cannot fit (test/test_eplace.cpp:115-179's overfull fixture, rebuilt):
    3,000 cells of 8 x 12 and 40 movable 208 x 208 macros heaped within +-20 of the centre of
    a 1,200 x 1,200 core of 100 rows, four fixed 60 x 60 terminals in the corners, and
    3-pin nets over the node list by the fixture's stride rule (node i, (7i + 3) mod movable,
    (13i + 11) mod nodes; pins at (+w/4, -h/4) of their node). Movable area is about 1.4x the
    core, so tau has a floor near 0.286 and the 0.10 target is out of reach: mGP stagnates.
    Start positions are seeded uniform draws (the fixture's own RNG is not needed: the device
    and the reference build are given the same PlaceDB)."""
    rng = np.random.default_rng(seed)
    core, row_h = 1200.0, 12.0
    c = 0.5 * core
    nodes = []
    for _ in range(3000):
        x, y = rng.uniform(-20.0, 20.0, 2)
        nodes.append((c + x, c + y, 8.0, row_h, 0))
    for _ in range(40):
        x, y = rng.uniform(-20.0, 20.0, 2)
        nodes.append((c + x, c + y, 208.0, 208.0, F_MACRO))
    for i in range(4):
        nodes.append((core - 40.0 if i % 2 else 40.0, core - 40.0 if i // 2 else 40.0, 60.0, 60.0, F_FIXED))
    n_mov, n_nodes = 3040, 3044
    nets, offs = [], []
    for i in range(n_mov):
        a, b, cc = i, (i * 7 + 3) % n_mov, (i * 13 + 11) % n_nodes
        if a == b or b == cc or a == cc:
            continue
        nets.append([a, b, cc])
        for nd in (a, b, cc):
            offs.append((np.float32(0.25) * np.float32(nodes[nd][2]), np.float32(-0.25) * np.float32(nodes[nd][3])))
    rows = [(r * row_h, row_h, 0.0, 1.0, int(core)) for r in range(int(core / row_h))]
    return make_db(nodes, rows, nets, offs, name="overfull")
