"""The iteration callback (EPlace::setIterCallback, src/gp/eplace.h:71-72) on the device loop
(GPU only).

The reference calls it after each iteration's metrics row with the PlaceDB at that iteration's
evaluation point (eplace.cpp:405-409); GlobalPlaceStage samples it every frame_stride
iterations for its frame hook (gp_stage.cpp:87-93). Here the device loop pauses after the row
of every iteration with iter % stride == 0 and hands the host every node's position at that
point. Checked:

  * the callback runs at exactly iterations 0, stride, 2*stride, ... of the stage (iteration 0
    is evaluated at the stage's starting positions, as the reference's first step evaluates its
    look-ahead point before moving);
  * at each call, the HPWL of the handed positions is the metrics row's HPWL for that iteration,
    and the positions are inside the core;
  * the stage's result (iterations, HPWL, overflow, delivered positions) is the same bit for bit
    with and without the callback, in the graph loop and in the host loop;
  * spg_eval_positions gives the last evaluation point (the last callback's positions with
    stride 1) and the one before it.
"""
import numpy as np
import pytest

from superplace_b200 import abi, engine

from .conftest import golden_small_db

pytestmark = pytest.mark.gpu


def run(stride=0, stage=abi.STAGE_MGP, host_loop=False, monkeypatch=None):
    if host_loop:
        monkeypatch.setenv("SPG_HOST_LOOP", "1")
    db, _ = golden_small_db(True)
    ep = engine.EPlace(db, abi.default_params(gp_bin_dim=64))
    calls = []
    if stride:
        ep.set_iter_callback(lambda st, it, x, y: calls.append((st, it, x, y)), stride)
    r = ep.run(stage)
    rows = ep.ctx.metrics(max(r.iterations, 1))
    return db, ep, r, rows, calls


def hpwl_at(db, x, y):
    ctx = engine.GpContext(db, abi.default_params(gp_bin_dim=64))
    ctx.set_positions(x, y)
    h = ctx.hpwl()
    ctx.close()
    return h


@pytest.mark.parametrize("stride", [1, 7])
def test_callback_iterations_and_points(stride):
    db, ep, r, rows, calls = run(stride)
    assert [c[1] for c in calls] == list(range(0, r.iterations, stride))
    assert all(c[0] == abi.STAGE_MGP for c in calls)
    lx, ly, hx, hy = db.core
    m = slice(0, db.num_movable)
    for _, it, x, y in calls[:: max(1, len(calls) // 6)]:
        h = hpwl_at(db, x, y)
        assert abs(h - rows["hpwl"][it]) <= 1e-12 * rows["hpwl"][it], (it, h, rows["hpwl"][it])
        assert np.all(x[m] - 0.5 * db.node_w[m] >= lx - 0.01) and np.all(x[m] + 0.5 * db.node_w[m] <= hx + 0.01)
        assert np.all(y[m] - 0.5 * db.node_h[m] >= ly - 0.01) and np.all(y[m] + 0.5 * db.node_h[m] <= hy + 0.01)
    if stride == 1:
        ex, ey = ep.ctx.eval_positions(0)
        assert np.array_equal(ex, calls[-1][2]) and np.array_equal(ey, calls[-1][3])
        px, py = ep.ctx.eval_positions(1)
        assert np.array_equal(px, calls[-2][2]) and np.array_equal(py, calls[-2][3])


@pytest.mark.parametrize("host_loop", [False, True])
def test_callback_leaves_the_placement_unchanged(host_loop, monkeypatch):
    db0, _, r0, _, _ = run(0, host_loop=host_loop, monkeypatch=monkeypatch)
    db1, _, r1, _, calls = run(3, host_loop=host_loop, monkeypatch=monkeypatch)
    assert len(calls) == (r1.iterations + 2) // 3
    assert (r0.iterations, r0.hpwl, r0.overflow) == (r1.iterations, r1.hpwl, r1.overflow)
    assert np.array_equal(db0.node_x, db1.node_x) and np.array_equal(db0.node_y, db1.node_y)


def test_callback_in_filler_only_moves_only_fillers():
    db, _ = golden_small_db(True)
    ep = engine.EPlace(db, abi.default_params(gp_bin_dim=64))
    ep.run(abi.STAGE_MGP)
    x0, y0 = db.node_x.copy(), db.node_y.copy()
    calls = []
    ep.set_iter_callback(lambda st, it, x, y: calls.append((st, it, x, y)), 5)
    r = ep.run(abi.STAGE_FILLER_ONLY)
    assert [c[1] for c in calls] == list(range(0, r.iterations, 5))
    n = db.num_nodes
    for st, it, x, y in calls:
        assert st == abi.STAGE_FILLER_ONLY
        assert np.array_equal(x[:n], x0[:n]) and np.array_equal(y[:n], y0[:n])
        # iteration 0 is evaluated where the stage starts; later points have moved the fillers
        assert np.array_equal(x[n:], x0[n:]) == (it == 0)


def test_eval_positions_needs_a_stage():
    db, _ = golden_small_db(True)
    ctx = engine.GpContext(db, abi.default_params(gp_bin_dim=64))
    with pytest.raises(engine.SpgError):
        ctx.eval_positions(0)
    ctx.close()


def test_global_place_frame_marks():
    """GlobalPlaceStage's frame marks (gp_stage.cpp:73-93,136) through flow.global_place: every
    frame_stride-th iteration of mGP, FILLERONLY and cGP on the accumulated clock t, the ends of
    mGP and cGP, and the mLG jump (here a stand-in legaliser that freezes the macros in place)."""
    from superplace_b200 import flow, generator
    from superplace_b200.placedb import F_FIXED

    db = generator.mixed_design(1002, n_cells=3000)

    def freeze(d):
        m = flow.movable_macros(d)
        d.node_flags[m] |= F_FIXED
        return {"macros": int(m.size)}

    marks = []
    res = flow.global_place(db, abi.default_params(gp_bin_dim=64), legalize_macros=freeze,
                            frame_hook=lambda m, x, y: marks.append((m, x.size)), frame_stride=10)
    n_mgp, n_fo, n_cgp = res["mGP"].iterations, res["FILLERONLY"].iterations, res["cGP"].iterations
    want = [("mGP", i, float(i), False) for i in range(0, n_mgp, 10)]
    want.append(("mGP", n_mgp, float(n_mgp), bool(res["mGP"].stagnated)))
    want.append(("mLG", -1, float(n_mgp), True))
    want += [("FILLERONLY", i, float(n_mgp + i), False) for i in range(0, n_fo, 10)]
    want += [("cGP", i, float(n_mgp + n_fo + i), False) for i in range(0, n_cgp, 10)]
    want.append(("cGP", n_cgp, float(n_mgp + n_fo + n_cgp), bool(res["cGP"].stagnated)))
    assert [(m.stage, m.iter, m.t, m.break_before) for m, _ in marks] == want
    assert all(n == db.total_nodes for _, n in marks)
