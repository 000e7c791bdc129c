"""GP diagnostics (--gp-diagnostics) from the device engine against the reference's own writer
(GPU only).

  * delivered point, same inputs: superplace_b200.diagnostics.write_gp_diagnostic and the
    reference build's diagnoseDelivered (src/gp/diagnostics.cpp:175-191, run through
    oracle/_ref) at the same positions, lambda, gamma and previous point write the same files:
    the same headers, rows and keys; geometry.csv byte for byte; the grid, bin rectangles,
    capacities, terminal and base charge, node identities, sizes, preconditioners and
    movements as the same text; the movable charge, potential, field, WA gradient, force and
    the probes within stated tolerances (the density maps are fixed point here and float sums
    there, the Poisson solve a different arithmetic); the overflow components the same but for
    bins whose excess is within rounding of zero;
  * a stage run with diagnostics on writes first_eval, last_eval and delivered (and
    stagnation_mid on the reference's overfull fixture, at the iteration where the stagnation
    counter first reaches half the window, replayed from the metrics rows by eplace.cpp's rule),
    with the metrics rows' lambda, gamma and step, and leaves the placement unchanged bit for
    bit; its first_eval matches the reference run's first_eval within tolerance.
"""
import csv
import json
import os

import numpy as np
import pytest

from superplace_b200 import abi, diagnostics, engine

from .checks import overfull_design
from .conftest import golden_small_db

pytestmark = pytest.mark.gpu

FILES = ("bins.csv", "nodes.csv", "geometry.csv", "metadata.json")


def ref_available():
    from oracle import ref

    if not ref.available():
        pytest.skip("oracle/_ref/libspref.so not built")
    return ref


def read_csv(path):
    with open(path) as f:
        rows = list(csv.reader(f))
    return rows[0], rows[1:]


def column(rows, header, name, kind=float):
    j = header.index(name)
    return np.array([kind(r[j]) for r in rows])


def close(a, b, rel):
    scale = max(np.abs(b).max(), 1e-30)
    return np.abs(a - b).max() <= rel * scale


def compare_point(ours, theirs, rel_maps=1e-4, rel_field=1e-3):
    for f in FILES:
        assert os.path.exists(os.path.join(ours, f)) and os.path.exists(os.path.join(theirs, f)), f
    with open(os.path.join(ours, "geometry.csv")) as a, open(os.path.join(theirs, "geometry.csv")) as b:
        assert a.read() == b.read()
    hb, rb = read_csv(os.path.join(ours, "bins.csv"))
    hr, rr = read_csv(os.path.join(theirs, "bins.csv"))
    assert hb == hr and len(rb) == len(rr)
    for name in ("bx", "by", "lx", "ly", "hx", "hy", "capacity", "terminal_charge", "base_charge"):
        assert [r[hb.index(name)] for r in rb] == [r[hr.index(name)] for r in rr], name
    for name in ("node_charge", "filler_charge", "overflow_area", "static_overflow_area"):
        assert close(column(rb, hb, name), column(rr, hr, name), rel_maps), name
    for name in ("potential", "field_x", "field_y"):
        assert close(column(rb, hb, name), column(rr, hr, name), rel_field), name
    cb, cr = column(rb, hb, "component", int), column(rr, hr, "component", int)
    assert np.mean((cb >= 0) == (cr >= 0)) > 0.99
    hn, rn = read_csv(os.path.join(ours, "nodes.csv"))
    hrn, rrn = read_csv(os.path.join(theirs, "nodes.csv"))
    assert hn == hrn and len(rn) == len(rrn)
    for name in ("id", "name", "filler", "macro", "x", "y", "width", "height", "preconditioner", "actual_dx",
                 "actual_dy", "boundary"):
        assert [r[hn.index(name)] for r in rn] == [r[hrn.index(name)] for r in rrn], name
    for name in ("wl_x", "wl_y"):
        assert close(column(rn, hn, name), column(rrn, hrn, name), 1e-5), name
    for name in ("force_x", "force_y", "gradient_x", "gradient_y"):
        assert close(column(rn, hn, name), column(rrn, hrn, name), rel_field), name
    assert np.mean(column(rn, hn, "component", int) == column(rrn, hrn, "component", int)) > 0.98
    mo = json.load(open(os.path.join(ours, "metadata.json")))
    mr = json.load(open(os.path.join(theirs, "metadata.json")))
    assert sorted(mo) == sorted(mr)
    for k in ("stage", "point", "iter", "movement_reference", "grid_dim", "origin", "bin_step",
              "overflow_denominator", "eval_lambda", "eval_gamma", "step_size"):
        assert mo[k] == mr[k], k
    for k in ("overflow", "overflow_area", "energy"):
        assert abs(mo[k] - mr[k]) <= 1e-3 * abs(mr[k]) + 1e-9, (k, mo[k], mr[k])
    assert abs(mo["static_overflow_area"] - mr["static_overflow_area"]) <= 1e-3 * max(mr["overflow_area"], 1.0)
    assert abs(len(mo["components"]) - len(mr["components"])) <= max(2, len(mr["components"]) // 20)
    assert [(p["direction"], p["fraction_of_bin"]) for p in mo["probes"]] == \
        [(p["direction"], p["fraction_of_bin"]) for p in mr["probes"]]
    for po, pr in zip(mo["probes"], mr["probes"]):
        assert abs(po["overflow"] - pr["overflow"]) <= 2e-3 * abs(pr["overflow"]) + 1e-6
        assert abs(po["energy"] - pr["energy"]) <= 2e-3 * abs(pr["energy"])
    return mo


def test_delivered_point_matches_reference_writer(tmp_path):
    ref = ref_available()
    db, _ = golden_small_db(True)
    params = abi.default_params(gp_bin_dim=64)
    ep = engine.EPlace(db, params)
    r = ep.run(abi.STAGE_MGP)
    rows = ep.ctx.metrics()
    last = r.iterations - 1
    lx, ly = ep.ctx.eval_positions(0)
    idx = diagnostics.opt_index(db, abi.STAGE_MGP)
    prev = np.concatenate([lx[idx], ly[idx]])
    lam, gam = float(rows["eval_lambda"][last]), float(rows["eval_gamma"][last])
    ours = diagnostics.write_gp_diagnostic(str(tmp_path / "ours"), abi.STAGE_MGP, "delivered", last, lam, gam, 0.0,
                                           db, params, 64, db.node_x, db.node_y, prev)
    ref.RefDb(db).diagnose_delivered(params, tmp_path / "ref", abi.STAGE_MGP, last, lam, gam, 64, prev)
    compare_point(ours, str(tmp_path / "ref" / "diagnostics" / "mGP" / "delivered"))


def test_stage_run_writes_the_points(tmp_path):
    ref = ref_available()
    db, _ = golden_small_db(True)
    db0 = db.copy()
    params = abi.default_params(gp_bin_dim=64)
    ep = engine.EPlace(db, params)
    r = ep.run(abi.STAGE_MGP, diagnostics=str(tmp_path / "ours"))
    rows = ep.ctx.metrics()
    base = tmp_path / "ours" / "diagnostics" / "mGP"
    assert sorted(os.listdir(base)) == ["delivered", "first_eval", "last_eval"]
    for point, it in (("first_eval", 0), ("last_eval", r.iterations - 1), ("delivered", r.iterations - 1)):
        meta = json.load(open(base / point / "metadata.json"))
        assert meta["iter"] == it and meta["point"] == point
        assert meta["eval_lambda"] == float(np.float32(rows["eval_lambda"][it]))
        assert meta["eval_gamma"] == float(np.float32(rows["eval_gamma"][it]))
        step = 0.0 if point == "delivered" else float(np.float32(rows["step_size"][it]))
        assert meta["step_size"] == step
        _, nodes = read_csv(base / point / "nodes.csv")
        assert len(nodes) == diagnostics.opt_index(db, abi.STAGE_MGP).size
    # the same placement as without diagnostics
    plain = engine.EPlace(db0, params)
    r0 = plain.run(abi.STAGE_MGP)
    assert (r0.iterations, r0.hpwl) == (r.iterations, r.hpwl)
    assert np.array_equal(db0.node_x, db.node_x) and np.array_equal(db0.node_y, db.node_y)
    # against the reference's run of the same stage: its first_eval within tolerance
    rdb, _ = golden_small_db(True)
    ref.RefDb(rdb).eplace_diagnostics(params, tmp_path / "ref", abi.STAGE_MGP)
    mo = json.load(open(base / "first_eval" / "metadata.json"))
    mr = json.load(open(tmp_path / "ref" / "diagnostics" / "mGP" / "first_eval" / "metadata.json"))
    assert sorted(mo) == sorted(mr)
    for k in ("eval_lambda", "eval_gamma", "step_size", "overflow", "energy"):
        assert abs(mo[k] - mr[k]) <= 1e-3 * abs(mr[k]), (k, mo[k], mr[k])


def stagnation_mid_row(tau, window, gain):
    """The iteration where eplace.cpp's counter of iterations without enough overflow gain first
    reaches max(1, window / 2) (eplace.cpp:421-433), replayed from the rows' tau in float."""
    ref = np.float32(np.inf)
    since = 0
    for i, t in enumerate(np.asarray(tau, np.float32)):
        if t < np.float32(ref * np.float32(np.float32(1.0) - np.float32(gain))):
            ref, since = t, 0
        else:
            since += 1
        if since >= max(1, window // 2):
            return i
    return None


def test_stagnation_mid_point(tmp_path):
    db = overfull_design(7)
    engine.initialize_fillers(db, 1.0, 1002)
    params = abi.default_params(gp_max_iter=500, gp_stagnation_window=40)
    ep = engine.EPlace(db, params)
    r = ep.run(abi.STAGE_MGP, diagnostics=str(tmp_path))
    assert r.stagnated
    rows = ep.ctx.metrics()
    expect = stagnation_mid_row(rows["overflow"], 40, params.gp_stagnation_min_gain)
    assert expect is not None
    meta = json.load(open(tmp_path / "diagnostics" / "mGP" / "stagnation_mid" / "metadata.json"))
    assert meta["iter"] == expect
    assert meta["eval_lambda"] == float(np.float32(rows["eval_lambda"][expect]))
    delivered = json.load(open(tmp_path / "diagnostics" / "mGP" / "delivered" / "metadata.json"))
    assert delivered["iter"] == r.rollback_iter
