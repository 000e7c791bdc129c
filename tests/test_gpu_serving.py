"""Placement serving on the device (GPU only): every request's result is the same alone and in
the mix. Requests of 1k-20k cells (64x64 grids with the FP32 Poisson, 128x128 with the split-BF16
one) are placed one at a time, then concurrently with four slots; each request's placement,
iteration count and HPWL must be identical bit for bit, and every one must converge."""
import numpy as np
import pytest

from superplace_b200 import engine, generator, serving

pytestmark = pytest.mark.gpu

CELLS = [1000, 2500, 20000, 1500, 4000, 18000]


@pytest.fixture(scope="module")
def requests():
    out = []
    for i, n in enumerate(CELLS):
        db, grid = generator.scaled_design(300 + i, n)
        engine.initialize_fillers(db, 1.0, 1002)
        out.append((db, grid))
    assert {g for _, g in out} == {64, 128}
    return out


def place_all(requests, slots):
    with serving.PlacementServer(slots=slots) as srv:
        futs = [srv.submit(db, g) for db, g in requests]
        res = [f.result(timeout=600) for f in futs]
    return res, srv.peak_running


def test_reloaded_context_matches_a_fresh_one(requests):
    """spg_ctx_load: a context that placed a larger netlist, reloaded with a smaller one (its
    buffers reused at their old capacity, its loop graph updated) places it exactly as a fresh
    context does."""
    from superplace_b200 import abi

    (big, gb), (small, gs) = requests[2], requests[0]
    pb = abi.default_params(gp_bin_dim=gb, poisson_precision=serving.choose_precision(gb, "auto"))
    ps = abi.default_params(gp_bin_dim=gs, poisson_precision=serving.choose_precision(gs, "auto"))

    def run(ctx, db):
        ctx.set_positions(db.node_x, db.node_y)
        ctx.set_flags(db.node_flags)
        r = ctx.run(abi.STAGE_MGP)
        return r, ctx.positions()

    fresh = engine.GpContext(small, ps)
    rf, (xf, yf) = run(fresh, small)
    fresh.close()
    ctx = engine.GpContext(big, pb)
    run(ctx, big)
    ctx.load(small, ps)
    rr, (xr, yr) = run(ctx, small)
    ctx.load(small, ps)  # and again, onto a context already holding this netlist
    r2, (x2, y2) = run(ctx, small)
    ctx.close()
    for r, x, y in ((rr, xr, yr), (r2, x2, y2)):
        assert r.converged == 1 and r.iterations == rf.iterations and r.hpwl == rf.hpwl
        assert np.array_equal(x, xf) and np.array_equal(y, yf)


def test_context_alternating_grid_sizes_matches_fresh_contexts(requests):
    """One context places a 64x64-grid request, a 128x128 one, then the first again: each grid
    size keeps its own Poisson plan and loop graph, and a later netlist patches the kept
    graph's kernel arguments. Every placement equals a fresh context's bit for bit."""
    from superplace_b200 import abi

    order = [requests[0], requests[2], requests[1], requests[0]]
    assert [g for _, g in order] == [64, 128, 64, 64]

    def run(ctx, db):
        ctx.set_positions(db.node_x, db.node_y)
        ctx.set_flags(db.node_flags)
        r = ctx.run(abi.STAGE_MGP)
        return r, ctx.positions()

    def params(g):
        return abi.default_params(gp_bin_dim=g, poisson_precision=serving.choose_precision(g, "auto"))

    fresh = []
    for db, g in order:
        c = engine.GpContext(db, params(g))
        fresh.append(run(c, db))
        c.close()
    ctx = None
    for (db, g), (rf, (xf, yf)) in zip(order, fresh):
        if ctx is None:
            ctx = engine.GpContext(db, params(g))
        else:
            ctx.load(db, params(g))
        r, (x, y) = run(ctx, db)
        assert r.converged == 1 and r.iterations == rf.iterations and r.hpwl == rf.hpwl
        assert np.array_equal(x, xf) and np.array_equal(y, yf)
    ctx.close()


def test_same_result_alone_and_in_the_mix(requests):
    alone, _ = place_all(requests, 1)
    mix, peak = place_all(requests, 4)
    assert peak > 1  # the mix really ran requests side by side
    for a, b in zip(alone, mix):
        assert a.request_id == b.request_id
        assert a.result.converged == 1 and b.result.converged == 1
        assert a.result.iterations == b.result.iterations
        assert a.result.hpwl == b.result.hpwl
        assert np.array_equal(a.x, b.x) and np.array_equal(a.y, b.y)
