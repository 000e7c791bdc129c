"""The stage loop's Nesterov optimizer on the device, driven on the reference's own optimizer
test objective f(x) = 0.5 * sum c_i (x_i - t_i)^2 (test/test_nesterov.cpp:14-27) through
spg_nesterov_quadratic: the loop's step kernel, backtracking test and step decisions without a
placement around them.

Known answers pinned here, each as test/test_nesterov.cpp states it:
  * a first step 50x the safe one is pulled back by exactly one re-evaluation, and the
    look-ahead objective after three steps is tiny with backtracking and huge without
    (testBacktrackRecoversFromHugeStep, :189-218);
  * with a safe step backtracking changes nothing, bit for bit, evaluations included
    (testBacktrackIsNoopWhenStepIsSafe, :221-239);
  * an ill-conditioned problem converges with backtracking and reruns bit for bit
    (testBacktrackConverges, :151-182).
The same runs are compared with the reference's optimizer: the committed known answers of
tests/golden/nesterov.npz, and the reference build (oracle/_ref) live where it is present.
Device and reference differ only in the order of the FP64 norm sums (fixed trees on both
sides), so evaluation counts agree exactly and positions and objectives to float rounding.
"""
import numpy as np
import pytest

from superplace_b200 import engine

from .conftest import load_golden

pytestmark = pytest.mark.gpu


def huge_step(backtrack):
    n = 32
    coef = np.full(n, 4.0, np.float32)  # L = 4: the safe step is 0.25
    target = np.full(n, 3.0, np.float32)
    return engine.nesterov_quadratic(coef, target, np.zeros(n, np.float32), 3, backtrack=backtrack,
                                     init_step=50.0 / 4.0)


def iso(backtrack, steps=100):
    n = 64
    coef = np.full(n, 2.0, np.float32)
    target = (10.0 + 0.5 * np.arange(n)).astype(np.float32)
    return engine.nesterov_quadratic(coef, target, np.zeros(n, np.float32), steps, backtrack=backtrack)


def test_backtrack_recovers_from_huge_step():
    pos_bt, obj_bt, ev_bt, _, redo_bt = huge_step(True)
    pos_p, obj_p, ev_p, _, redo_p = huge_step(False)
    assert obj_bt < 1e-6
    assert obj_p > 1e3
    assert ev_bt == ev_p + 1  # exactly one re-evaluation
    assert (redo_bt, redo_p) == (1, 0)
    g = load_golden("nesterov.npz")
    for bt, pos, obj, ev in ((1, pos_bt, obj_bt, ev_bt), (0, pos_p, obj_p, ev_p)):
        meta = g[f"huge_bt{bt}_meta"]
        assert ev == int(meta[1])
        assert obj == pytest.approx(meta[0], rel=1e-5, abs=1e-9)
        np.testing.assert_allclose(pos, g[f"huge_bt{bt}_pos"], rtol=1e-5, atol=1e-6)


def test_backtrack_is_noop_when_step_is_safe():
    a, b = iso(True), iso(False)
    assert np.array_equal(a[0], b[0])  # bit for bit
    assert a[2] == b[2] and a[4] == 0
    g = load_golden("nesterov.npz")
    for bt, r in ((1, a), (0, b)):
        meta = g[f"iso_bt{bt}_meta"]
        assert r[2] == int(meta[1])
        np.testing.assert_allclose(r[0], g[f"iso_bt{bt}_pos"], rtol=1e-5)
        assert r[3] == pytest.approx(meta[2], rel=1e-4)  # the last step size


def test_backtrack_converges_and_reruns_bit_for_bit():
    n = 50
    i = np.arange(n)
    coef = (0.01 * np.power(10.0, 3.0 * i / (n - 1))).astype(np.float32)
    target = (-5.0 + 0.3 * i).astype(np.float32)
    start = np.full(n, 100.0, np.float32)
    d = start.astype(np.float64) - target
    obj0 = float(np.sum(0.5 * coef * d * d))
    a = engine.nesterov_quadratic(coef, target, start, 2000, backtrack=True)
    b = engine.nesterov_quadratic(coef, target, start, 2000, backtrack=True)
    assert a[1] < obj0 * 1e-6
    assert np.array_equal(a[0], b[0]) and a[2] == b[2] and a[1] == b[1]


@pytest.mark.parametrize("use_bb,backtrack,init_step", [(True, True, 0.0), (True, False, 0.0),
                                                        (False, True, 0.0), (True, True, 12.5)])
def test_matches_reference_optimizer(use_bb, backtrack, init_step):
    """Against the reference's NesterovOptimizer run live (oracle/_ref): the same step count
    from the same start on a mildly ill-conditioned quadratic; estimateInitialStep included
    when init_step is 0."""
    from oracle import ref

    if not ref.available():
        pytest.skip("oracle/_ref/libspref.so not built")
    rng = np.random.default_rng(5)
    n = 256
    coef = rng.uniform(0.5, 20.0, n).astype(np.float32)
    target = rng.uniform(-50.0, 50.0, n).astype(np.float32)
    start = rng.uniform(-100.0, 100.0, n).astype(np.float32)
    for steps in (1, 2, 5, 20):
        pos, obj, ev, step, _ = engine.nesterov_quadratic(coef, target, start, steps, use_bb=use_bb,
                                                          backtrack=backtrack, init_step=init_step)
        rpos, robj, rev, rstep = ref.nesterov_quadratic(coef, target, start, steps, use_bb=use_bb,
                                                        backtrack=backtrack, init_step=init_step)
        assert ev == rev, (steps, ev, rev)
        assert step == pytest.approx(rstep, rel=1e-5)
        assert obj == pytest.approx(robj, rel=1e-4, abs=1e-6)
        np.testing.assert_allclose(pos, rpos, rtol=1e-4, atol=1e-4 * np.abs(rpos).max())
