"""B2B quadratic initial placement (CPU): superplace_b200.qp against oracle/qp.py, the numpy
restatement of QuadraticPlacer (src/init/quadratic_placer.cpp) and forEachB2BPair
(src/init/b2b_model.h), and HPWL against the reference's own computeHPWL (oracle/_ref).

- The pair rule: test/test_b2b.cpp's identity. Along each axis sum w (pos_p - pos_q)^2 over a
  net's B2B pairs is that net's HPWL component, with 2P - 3 pairs. It is checked through the
  assembled matrix (x^T A x), and the same check fails on the oracle with the reference test's
  planted mistake.
- The linear system: CSR and right-hand side bit for bit against the oracle's float32 sums in
  the reference's order.
- The placement: final HPWL against the oracle's within tolerance (the solver's dot products
  are summed in another order), identical results for 1 and many threads, and the clamp and
  unconnected-node rules.
"""
import numpy as np
import pytest

from oracle import qp as oqp
from oracle import ref
from superplace_b200 import generator, qp
from superplace_b200.placedb import F_FIXED, make_db


def single_net_db(xs, ys):
    """test/test_b2b.cpp:36-58: one net over P movable 2x2 nodes, zero pin offsets."""
    nodes = [(float(x), float(y), 2.0, 2.0, 0) for x, y in zip(xs, ys)]
    return make_db(nodes, rows=[(0.0, 1000.0, 0.0, 1.0, 1000)], nets=[list(range(len(xs)))])


def quad_form(db, axis, pos):
    start, col, val, _ = qp.assemble(db, axis, params=qp.default_params(min_distance=1e-9))
    rows = np.repeat(np.arange(db.num_movable), np.diff(start))
    off = int(np.sum(col != rows))
    q = float(np.sum(val.astype(np.float64) * pos[rows].astype(np.float64) * pos[col].astype(np.float64)))
    return q, off // 2


def check_identity(xs, ys):
    xs, ys = np.asarray(xs, np.float32), np.asarray(ys, np.float32)
    db = single_net_db(xs, ys)
    P = len(xs)
    for axis, pos in ((0, xs), (1, ys)):
        q, pairs = quad_form(db, axis, pos)
        want = float(pos.max()) - float(pos.min())
        assert pairs == 2 * P - 3
        assert q == pytest.approx(want, rel=1e-3, abs=1e-3)


def test_b2b_identity_small_nets():
    check_identity([10, 50], [3, 90])
    check_identity([10, 30, 50], [90, 3, 40])
    check_identity([5, 12, 40, 7, 33], [1, 80, 22, 55, 9])
    check_identity([1, 20, 15, 40, 25], [50, 99, 2, 70, 60])  # extremes on different pins per axis


def test_b2b_identity_randomized():
    rng = np.random.default_rng(20260916)
    for _ in range(40):
        P = int(rng.integers(2, 11))
        check_identity(rng.uniform(0, 500, P), rng.uniform(0, 500, P))


def test_planted_mistake_breaks_identity():
    """The oracle with the p == lo test left out (test/test_b2b.cpp:159-196) loses pairs and
    the identity, so the identity check can tell."""
    xs = np.array([1, 20, 15, 40, 25], np.float32)
    db = single_net_db(xs, [50, 99, 2, 70, 60])
    lo, hi = oqp.bound_pins(db, db.node_x, db.node_y)[:2]
    good = oqp.b2b_pairs(db, 0, int(lo[0]), int(hi[0]), db.node_x, db.pin_offset_x, None, 1e-9)
    bad = oqp.b2b_pairs(db, 0, int(lo[0]), int(hi[0]), db.node_x, db.pin_offset_x, None, 1e-9,
                        drop_lower_bound_of_p=True)

    def form(pairs):
        return sum(float(w) * (float(db.node_x[p]) - float(db.node_x[q])) ** 2 for p, q, w in pairs)

    assert len(good) == 7 and form(good) == pytest.approx(39.0, rel=1e-4)
    assert len(bad) < 7 and abs(form(bad) - 39.0) > 1e-3


def qp_design(seed=5, n_cells=300, n_nets=330):
    """A small seeded design: fixed macros and pads, pin offsets, unit and non-unit net
    weights, a net above ignore_net_degree, a net with two pins on one node, an unconnected
    movable node, and random positions."""
    rng = np.random.default_rng(seed)
    w = rng.integers(2, 12, n_cells).astype(np.float32)
    db = generator.build_design(seed=seed, die=240.0, row_h=12.0, n_cells=n_cells, cell_w=w, n_nets=n_nets,
                                n_fixed_macros=2, fixed_cover=0.1, macro_rows=(2, 4), n_pads=12, name="qp")
    db.net_weight = rng.uniform(0.5, 3.0, db.num_nets).astype(np.float32)
    db.net_weight[rng.random(db.num_nets) < 0.7] = 1.0
    n = db.num_nodes
    db.node_x[: db.num_movable] = rng.uniform(db.core[0], db.core[2], db.num_movable).astype(np.float32)
    db.node_y[: db.num_movable] = rng.uniform(db.core[1], db.core[3], db.num_movable).astype(np.float32)
    assert n > db.num_movable  # fixed nodes present
    return db


def big_net_db(base):
    """base plus one net over 120 nodes (above ignore_net_degree) and one with two pins on one node."""
    db = base.copy()
    rng = np.random.default_rng(1)
    pin2node = list(db.pin2node)
    pin_net = list(db.pin2net)
    ox, oy = list(db.pin_offset_x), list(db.pin_offset_y)
    k = db.num_nets
    for nd in rng.choice(db.num_nodes, 120, replace=False):
        pin2node.append(int(nd)); pin_net.append(k); ox.append(0.5); oy.append(-0.5)
    for nd, o in ((3, 1.0), (3, -1.0), (7, 0.0)):
        pin2node.append(nd); pin_net.append(k + 1); ox.append(o); oy.append(o)
    db.pin2node = np.array(pin2node, np.int32)
    db.pin_offset_x, db.pin_offset_y = np.array(ox, np.float32), np.array(oy, np.float32)
    db.finalize_csr(np.array(pin_net, np.int32), k + 2)
    db.net_weight = np.concatenate([db.net_weight, [2.0, 1.5]]).astype(np.float32)
    db.extend_node2pin()
    return db


def test_assembly_bit_exact_against_oracle():
    db = big_net_db(qp_design())
    for axis in (0, 1):
        start, col, val, rhs = qp.assemble(db, axis)
        o_start, o_col, o_val, o_rhs = oqp.assemble(db, axis, db.node_x, db.node_y, db.net_weight)
        assert np.array_equal(start, o_start) and np.array_equal(col, o_col)
        assert np.array_equal(val.view(np.uint32), o_val.view(np.uint32))
        assert np.array_equal(rhs.view(np.uint32), o_rhs.view(np.uint32))
        rows = np.repeat(np.arange(db.num_movable), np.diff(start))
        assert np.all(np.diff(col)[np.diff(rows) == 0] > 0)  # ascending columns, no duplicates


def test_unconnected_node_gets_the_tiny_diagonal():
    db = qp_design()
    connected = np.zeros(db.num_nodes, bool)
    for k in range(db.num_nets):
        pins = db.flat_net2pin[db.net2pin_start[k]:db.net2pin_start[k + 1]]
        if 2 <= len(pins) <= 100:
            connected[db.pin2node[pins]] = True
    lonely = np.flatnonzero(~connected[: db.num_movable])
    assert lonely.size > 0
    start, col, val, rhs = qp.assemble(db, 0)
    for i in lonely[:5]:
        row = slice(start[i], start[i + 1])
        assert list(col[row]) == [i] and val[row][0] == np.float32(1e-6)
        assert rhs[i] == np.float32(np.float32(1e-6) * db.node_x[i])


@pytest.mark.skipif(not ref.available(), reason="oracle/_ref not built")
def test_host_hpwl_matches_reference():
    db = qp_design()
    assert qp.host_hpwl(db) == ref.RefDb(db).hpwl()


def test_place_matches_oracle():
    db = qp_design()
    a = db.copy()
    rows = qp.QuadraticPlacer().place(a)
    x, y, hist = oqp.place(db, db.net_weight)
    n = db.num_movable
    assert rows["iter"].shape[0] == len(hist)
    assert np.allclose(rows["hpwl"], hist, rtol=1e-4)  # every outer iteration
    # movable nodes inside the core; fixed nodes untouched
    assert np.all(a.node_x[:n] - a.node_w[:n] / 2 >= db.core[0] - 1e-3)
    assert np.all(a.node_x[:n] + a.node_w[:n] / 2 <= db.core[2] + 1e-3)
    assert np.array_equal(a.node_x[n:db.num_nodes], db.node_x[n:db.num_nodes])
    # the QP pulls the netlist together: HPWL well below that of the random start
    assert rows["hpwl"][-1] < 0.5 * qp.host_hpwl(db)
    assert np.abs(a.node_x[:n] - x[:n]).max() < 1e-3 * (db.core[2] - db.core[0])
    assert np.abs(a.node_y[:n] - y[:n]).max() < 1e-3 * (db.core[3] - db.core[1])


def test_place_independent_of_threads():
    db = big_net_db(qp_design(seed=9))
    out = []
    for threads in (1, 3, 8):
        a = db.copy()
        rows = qp.QuadraticPlacer(qp.default_params(threads=threads)).place(a)
        out.append((a.node_x.copy(), a.node_y.copy(), rows["hpwl"].copy()))
    for x, y, h in out[1:]:
        assert np.array_equal(x.view(np.uint32), out[0][0].view(np.uint32))
        assert np.array_equal(y.view(np.uint32), out[0][1].view(np.uint32))
        assert np.array_equal(h, out[0][2])


def test_outer_loop_stops_on_hpwl_stall_or_cap():
    db = qp_design()
    rows = qp.QuadraticPlacer(qp.default_params(max_iter=3)).place(db.copy())
    assert list(rows["iter"]) == [0, 1, 2]
    rows = qp.QuadraticPlacer(qp.default_params(outer_tol=0.5)).place(db.copy())
    assert list(rows["iter"]) == [0, 1, 2, 3, 4, 5]  # the stall test starts after the fifth


def test_wide_node_goes_to_the_core_centre_and_no_movable_is_a_no_op():
    nodes = [(10.0, 10.0, 500.0, 4.0, 0), (20.0, 20.0, 4.0, 4.0, 0), (90.0, 50.0, 4.0, 4.0, F_FIXED)]
    db = make_db(nodes, rows=[(0.0, 100.0, 0.0, 1.0, 100)], nets=[[0, 1, 2]])
    qp.QuadraticPlacer().place(db)
    assert db.node_x[0] == 50.0  # wider than the core
    assert db.node_x[2] == 90.0 and db.node_y[2] == 50.0
    only_fixed = make_db([(5.0, 5.0, 2.0, 2.0, F_FIXED)], rows=[(0.0, 10.0, 0.0, 1.0, 10)], nets=[[0]])
    rows = qp.QuadraticPlacer().place(only_fixed)
    assert rows["iter"].shape[0] == 0 and only_fixed.node_x[0] == 5.0


def test_device_solver_fails_loudly_without_a_gpu():
    from superplace_b200 import engine
    if engine.device_available():
        pytest.skip("a GPU is present")
    with pytest.raises(engine.SpgError) as e:
        qp.QuadraticPlacer(qp.default_params(device=1)).place(qp_design())
    assert e.value.code == -2  # SPG_E_NO_DEVICE, no host fallback


@pytest.mark.parametrize("ignore,min_distance", [(5, 1.0), (6, 10.0), (2, 0.25)])
def test_assembly_degree_cap_and_distance_floor(ignore, min_distance):
    """Nets of degree exactly ignore_net_degree are kept and one above is dropped
    (src/init/quadratic_placer.cpp:84); a large qp_min_distance floors the weight denominator."""
    db = big_net_db(qp_design(seed=11))
    p = qp.default_params(ignore_net_degree=ignore, min_distance=min_distance)
    degs = np.diff(db.net2pin_start)
    assert np.any(degs == ignore) and np.any(degs == ignore + 1)
    for axis in (0, 1):
        start, col, val, rhs = qp.assemble(db, axis, params=p)
        o = oqp.assemble(db, axis, db.node_x, db.node_y, db.net_weight, min_distance=min_distance,
                         ignore_net_degree=ignore)
        assert np.array_equal(start, o[0]) and np.array_equal(col, o[1])
        assert np.array_equal(val.view(np.uint32), o[2].view(np.uint32))
        assert np.array_equal(rhs.view(np.uint32), o[3].view(np.uint32))
