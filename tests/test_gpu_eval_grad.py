"""EPlace::Impl::objAndGrad (src/gp/eplace.cpp:136-203) on the device against the reference.

spg_eval_grad runs the stage loop's own kernels (the loop body with no step applied: the step
kernel's fixed-point scatter, WA pass 1 with HPWL and the cells' WA pass 2, rho and tau, the
Poisson solve, the large nodes' gather, and the fused assembly with the cell gather and
preconditioning) at
caller positions. The reference side is objAndGrad's composition of the reference's own
operators (oracle/_ref: BinGrid, WaWirelength, computeHPWL and the assembly of
eplace.cpp:166-189). Both evaluate the same opt set at the same positions with the same
lambda and gamma.

Tolerances, from the arithmetic each side does:
  * HPWL: FP32 bounding boxes summed in FP64 on both sides, in different fixed orders: 1e-9.
  * tau: the device's density maps are exact integer sums of the reference's FP32 overlap
    products; the reference adds the same products in FP32 in its own order: 1e-5.
  * WA value: FP32 exponentials, FP64 sum: 1e-6.
  * gradient: max |diff| within 1e-5 of max |grad| with the plain FP32 Poisson and the FP64
    form alike (the reference's solve is an FP32 FFT, so the bound is set by the FP32 field
    on both sides); sum |dWL| within 1e-6 and sum |q xi| within 1e-5 relative.
The mixed design has 10 movable macros whose footprints exceed 16 bins: their force is the
block-per-node gather, summed as a fixed tree rather than in the reference's order, and is
held to the same bound.
"""
import numpy as np
import pytest

from superplace_b200 import abi, engine, generator

from .conftest import golden_small_db
from .test_gpu_stages import mixed_small

pytestmark = pytest.mark.gpu

BINS = 64


def opt_positions(db, stage):
    """buildOptSet's order (eplace.cpp:82-94) over db's current positions, x then y."""
    from superplace_b200.placedb import F_FIXED, F_MACRO, F_NI

    f = db.node_flags
    if stage == abi.STAGE_FILLER_ONLY:
        cells = np.zeros(0, np.int64)
    else:
        m = np.arange(db.num_movable)
        keep = (f[m] & (F_FIXED | F_NI)) == 0
        if stage == abi.STAGE_CGP:
            keep &= (f[m] & F_MACRO) == 0
        cells = m[keep]
    idx = np.concatenate([cells, np.arange(db.num_nodes, db.total_nodes)])
    return np.concatenate([db.node_x[idx], db.node_y[idx]]).astype(np.float32), idx


def compare(db, stage, precision, lam=None, gamma=None, tol_grad=1e-5):
    from oracle import ref

    if not ref.available():
        pytest.skip("oracle/_ref/libspref.so not built")
    params = abi.default_params(gp_bin_dim=BINS, poisson_precision=precision)
    ctx = engine.GpContext(db, params)
    ctx.set_positions()
    ctx.set_flags(db.node_flags)
    pos, idx = opt_positions(db, stage)
    assert ctx.n_opt(stage) * 2 == pos.size
    rdb = ref.RefDb(db)
    assert rdb.n_opt(params, stage) * 2 == pos.size
    if lam is None:  # the lambda_0 probe's values (eplace.cpp:248-259), from the reference
        g1 = ref.gamma(1.0, ctx.grid_info()["step_x"])
        _, probe = rdb.obj_and_grad(params, stage, 1.0, g1, pos)
        lam = probe["sum_wl"] / probe["sum_den"] if probe["sum_den"] > 0 else 1.0
        if not lam > 0:  # eplace.cpp:257 (FILLERONLY: no wirelength term)
            lam = 1.0
        gamma = ref.gamma(probe["tau"], ctx.grid_info()["step_x"])
    got, gs = ctx.eval_grad(stage, lam, gamma, pos)
    want, ws = rdb.obj_and_grad(params, stage, lam, gamma, pos)
    assert gs["hpwl"] == pytest.approx(ws["hpwl"], rel=1e-9)
    assert gs["tau"] == pytest.approx(ws["tau"], rel=1e-5, abs=1e-7)
    assert gs["obj"] == pytest.approx(ws["obj"], rel=1e-6)
    assert gs["sum_wl"] == pytest.approx(ws["sum_wl"], rel=1e-6)
    assert gs["sum_den"] == pytest.approx(ws["sum_den"], rel=1e-5)
    scale = np.abs(want).max()
    err = np.abs(got.astype(np.float64) - want).max() / scale
    assert err <= tol_grad, err
    return got, want, idx, err


@pytest.mark.parametrize("precision", [abi.POISSON_FP32, abi.POISSON_FP64])
def test_mgp_gradient_at_start(small, precision):
    db, _ = golden_small_db(True)
    compare(db, abi.STAGE_MGP, precision)


@pytest.mark.parametrize("precision", [abi.POISSON_FP32, abi.POISSON_FP64])
def test_mgp_gradient_at_spread_placement(precision):
    """At the reference's own final mGP placement (tests/golden: mgp_x, mgp_y), where the
    field is smooth and the wirelength term dominates."""
    db, g = golden_small_db(True)
    db.node_x[:] = g["mgp_x"]
    db.node_y[:] = g["mgp_y"]
    compare(db, abi.STAGE_MGP, precision)


def test_mixed_size_gradient_with_large_nodes():
    db = mixed_small()
    got, want, idx, _ = compare(db, abi.STAGE_MGP, abi.POISSON_FP32)
    from superplace_b200.placedb import F_MACRO

    macro_k = np.nonzero((db.node_flags[idx] & F_MACRO) != 0)[0]
    assert macro_k.size == 10
    n = idx.size
    k = np.concatenate([macro_k, n + macro_k])
    assert np.abs(got[k] - want[k]).max() <= 1e-5 * np.abs(want).max()


def test_filler_only_and_cgp_opt_sets():
    """FILLERONLY (fillers only) and cGP (no macros) after the macros are frozen."""
    from superplace_b200.placedb import F_FIXED, F_MACRO

    db = mixed_small()
    m = (db.node_flags[: db.num_movable] & F_MACRO) != 0
    db.node_flags[: db.num_movable][m] |= F_FIXED
    for stage in (abi.STAGE_FILLER_ONLY, abi.STAGE_CGP):
        compare(db.copy(), stage, abi.POISSON_FP32)


def test_loop_evaluation_matches_stage_first_row():
    """The hook and the stage loop run the same kernels: at the stage's start positions with
    the lambda and gamma of the stage's first evaluation, the hook's HPWL, tau and both
    gradient-norm sums are the first metrics row's, bit for bit."""
    db, _ = golden_small_db(True)
    params = abi.default_params(gp_bin_dim=BINS)
    ep = engine.EPlace(db.copy(), params)
    r = ep.run(abi.STAGE_MGP)
    rows = ep.ctx.metrics()
    ctx = engine.GpContext(db, params)
    ctx.set_positions()
    pos, _ = opt_positions(db, abi.STAGE_MGP)
    # the stage clamps the start into the core before its first evaluation (eplace.cpp:240-244)
    lx, ly, hx, hy = db.core
    n = pos.size // 2
    _, idx = opt_positions(db, abi.STAGE_MGP)
    hw, hh = 0.5 * db.node_w[idx], 0.5 * db.node_h[idx]
    xlo = np.float32(lx) + hw + np.float32(1e-3)
    xhi = np.maximum(xlo, np.float32(hx) - hw - np.float32(1e-3))
    ylo = np.float32(ly) + hh + np.float32(1e-3)
    yhi = np.maximum(ylo, np.float32(hy) - hh - np.float32(1e-3))
    pos[:n] = np.minimum(np.maximum(pos[:n], xlo), xhi)
    pos[n:] = np.minimum(np.maximum(pos[n:], ylo), yhi)
    _, s = ctx.eval_grad(abi.STAGE_MGP, rows["eval_lambda"][0], rows["eval_gamma"][0], pos)
    assert r.iterations > 0
    assert s["hpwl"] == rows["hpwl"][0]
    assert np.float32(s["tau"]) == np.float32(rows["overflow"][0])
    assert np.float32(s["sum_wl"]) == np.float32(rows["grad_norm_wl"][0])
    assert np.float32(s["sum_den"]) == np.float32(rows["grad_norm_den"][0])
