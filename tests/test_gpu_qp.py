"""The QP's BiCGSTAB on the GPU (qp_device.cu) against the host solver (the same summation
order on both sides, so the placements agree bit for bit) and directly against the oracle."""
import numpy as np
import pytest

from superplace_b200 import generator, qp

from .test_qp import big_net_db, qp_design

pytestmark = pytest.mark.gpu


def run(db, **kw):
    a = db.copy()
    rows = qp.QuadraticPlacer(qp.default_params(**kw)).place(a)
    return a, rows


@pytest.mark.parametrize("make", [lambda: qp_design(), lambda: big_net_db(qp_design(seed=9)),
                                  lambda: generator.small_design(1002)])
def test_device_qp_matches_host_bit_for_bit(make):
    db = make()
    if not hasattr(db, "net_weight"):
        db.net_weight = np.ones(db.num_nets, np.float32)
    host, hrows = run(db, device=0)
    dev, drows = run(db, device=1)
    assert np.array_equal(dev.node_x.view(np.uint32), host.node_x.view(np.uint32))
    assert np.array_equal(dev.node_y.view(np.uint32), host.node_y.view(np.uint32))
    for k in ("iter", "solver_iters_x", "solver_iters_y", "hpwl"):
        assert np.array_equal(drows[k], hrows[k]), k
    assert np.array_equal(drows["err"].view(np.uint32), hrows["err"].view(np.uint32))


def test_device_qp_is_deterministic_and_handles_trivial_systems():
    db = qp_design()
    a, ra = run(db, device=1)
    b, rb = run(db, device=1)
    assert np.array_equal(a.node_x, b.node_x) and np.array_equal(ra["hpwl"], rb["hpwl"])
    # a design whose nets are all above ignore_net_degree: every row is the tiny diagonal
    c, rc = run(db, device=1, ignore_net_degree=1)
    h, rh = run(db, device=0, ignore_net_degree=1)
    assert np.array_equal(c.node_x, h.node_x) and np.array_equal(rc["hpwl"], rh["hpwl"])


def test_device_qp_matches_oracle():
    """The device solver directly against oracle/qp.py (numpy float32, the reference's order;
    its dot products are numpy's, so the bar is a tolerance): HPWL of every outer iteration
    within 1e-4 relative and positions within 1e-3 of the core size, as the host solver's CPU
    test holds them."""
    from oracle import qp as oqp

    db = qp_design()
    dev, rows = run(db, device=1)
    x, y, hist = oqp.place(db, db.net_weight)
    n = db.num_movable
    assert rows["iter"].shape[0] == len(hist)
    assert np.allclose(rows["hpwl"], hist, rtol=1e-4)
    assert np.abs(dev.node_x[:n] - x[:n]).max() < 1e-3 * (db.core[2] - db.core[0])
    assert np.abs(dev.node_y[:n] - y[:n]).max() < 1e-3 * (db.core[3] - db.core[1])
