"""Generates tests/golden/*.npz from the reference's OWN CPU code (oracle/_ref, built from
the reference sources by oracle/Makefile). Run here, where the reference is present:

    make -C oracle ref && python tests/golden/make_golden.py

The fixtures pin the oracle (tests/test_oracle.py) and, through it, the CUDA path. Each
file stores its inputs too, so the tests need neither the reference nor the generator.
"""
from __future__ import annotations

import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from oracle import ref  # noqa: E402
from superplace_b200 import abi, generator  # noqa: E402

OUT = os.path.dirname(os.path.abspath(__file__))

DB_KEYS = ("node_x", "node_y", "node_w", "node_h", "node_flags", "pin_offset_x", "pin_offset_y",
           "pin2node", "pin2net", "net2pin_start", "flat_net2pin", "node2pin_start",
           "flat_node2pin", "row_ly", "row_height", "row_lx", "row_step", "row_num_sites")


def db_arrays(db):
    d = {k: getattr(db, k) for k in DB_KEYS}
    d["counts"] = np.array([db.num_movable, db.num_nodes, db.num_fillers], np.int64)
    d["core"] = np.array(db.core, np.float32)
    d["row_height_mode"] = np.array(db.row_height_mode, np.float32)
    d["total_row_area"] = np.array(db.total_row_area, np.float64)
    return d


def small_with_fillers(seed=1002):
    db = generator.small_design(seed)
    r = ref.RefDb(db)
    info = r.fillers_init(1.0, seed)
    x, y, _, _, _ = r.nodes()
    db.set_fillers(int(info[0]), info[1], info[2], x[db.num_nodes:], y[db.num_nodes:])
    return db, r, info


def make_small():
    db0 = generator.small_design(1002)
    base = db_arrays(db0)
    db, r, info = small_with_fillers(1002)
    out = {("in_" + k): v for k, v in base.items()}
    out["filler_info"] = np.array(info, np.float64)
    out["filler_x"] = db.node_x[db.num_nodes:].copy()
    out["filler_y"] = db.node_y[db.num_nodes:].copy()
    for dim in (64, 32):
        g = ref.RefGrid(r, 1.0, dim)
        g.accumulate()
        g.solve()
        out[f"d{dim}_info"] = np.array([g.dim, g.step_x, g.step_y, g.origin_x, g.origin_y], np.float64)
        out[f"d{dim}_den"] = np.array(g.overflow_denominator, np.float64)
        out[f"d{dim}_terminal"] = g.read(2)
        out[f"d{dim}_base"] = g.read(3)
        out[f"d{dim}_node"] = g.read(0)
        out[f"d{dim}_filler"] = g.read(1)
        out[f"d{dim}_tau"] = np.array(g.overflow(), np.float32)
        out[f"d{dim}_charge"] = np.array(g.total_charge(), np.float64)
        out[f"d{dim}_xi_x"] = g.read(6)
        out[f"d{dim}_xi_y"] = g.read(7)
        out[f"d{dim}_force"] = g.gather()
    for gamma in (50.0, 5.0):
        wl, grad = r.wa(gamma, 100)
        out[f"wa{int(gamma)}_wl"] = np.array(wl, np.float64)
        out[f"wa{int(gamma)}_grad"] = grad
    out["hpwl"] = np.array(r.hpwl(), np.float64)
    taus = np.array([0.0, 0.05, 0.0999, 0.1, 0.3, 0.7, 1.0, 1.0001, 2.5], np.float32)
    out["gamma_tau"] = taus
    out["gamma_val"] = np.array([ref.gamma(float(t), 9.375) for t in taus], np.float32)
    # mGP trajectory of the reference on this instance (64x64 bins)
    r2 = ref.RefDb(db)
    res, rows = r2.eplace(abi.default_params(gp_bin_dim=64))
    out["mgp_result"] = np.array([res[k] for k in ("iterations", "hpwl", "overflow", "converged",
                                                   "stagnated", "rollback_iter", "evaluations")],
                                 np.float64)
    out["mgp_rows"] = rows[:, :7]
    x, y, _, _, _ = r2.nodes()
    out["mgp_x"], out["mgp_y"] = x, y
    np.savez_compressed(os.path.join(OUT, "small_design.npz"), **out)


def make_nesterov():
    """test/test_nesterov.cpp-style quadratics through the reference optimizer."""
    out = {}
    n = 64
    coef = np.full(n, 2.0, np.float32)
    target = (10.0 + 0.5 * np.arange(n)).astype(np.float32)
    for bt in (0, 1):
        pos, obj, ev, step = ref.nesterov_quadratic(coef, target, np.zeros(n, np.float32), 100,
                                                    use_bb=True, backtrack=bool(bt))
        out[f"iso_bt{bt}_pos"] = pos
        out[f"iso_bt{bt}_meta"] = np.array([obj, ev, step])
    coef4 = np.full(32, 4.0, np.float32)
    t3 = np.full(32, 3.0, np.float32)
    for bt in (0, 1):
        pos, obj, ev, step = ref.nesterov_quadratic(coef4, t3, np.zeros(32, np.float32), 3,
                                                    use_bb=True, backtrack=bool(bt),
                                                    init_step=50.0 / 4.0)
        out[f"huge_bt{bt}_pos"] = pos
        out[f"huge_bt{bt}_meta"] = np.array([obj, ev, step])
    np.savez_compressed(os.path.join(OUT, "nesterov.npz"), **out)


if __name__ == "__main__":
    make_small()
    make_nesterov()
    for f in sorted(os.listdir(OUT)):
        if f.endswith(".npz"):
            print(f, os.path.getsize(os.path.join(OUT, f)))
