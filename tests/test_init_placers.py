"""The random and cluster initial placers (CPU) against the reference's own RandomPlacer and
ClusterPlacer (src/init/random_placer.cpp, src/init/cluster_common.cpp, cluster_fc.cpp,
cluster_bc.cpp, compiled from their sources into oracle/_ref): positions bit for bit."""
import numpy as np
import pytest

from oracle import ref
from superplace_b200 import generator
from superplace_b200.initial import METHODS, make_initial_placer
from superplace_b200.placedb import make_db

needs_ref = pytest.mark.skipif(not ref.available(), reason="oracle/_ref not built")


def compare(db, method, **kw):
    mine = db.copy()
    rep = make_initial_placer(method, **kw).place(mine)
    r = ref.RefDb(db)
    ref.init_place(r, method, kw.get("seed", 1002), kw.get("cluster_target_count", 0), kw.get("ignore_net_degree", 100))
    x, y = r.nodes()[:2]
    n = db.num_nodes
    assert np.array_equal(mine.node_x[:n].view(np.uint32), x[:n].view(np.uint32)), method
    assert np.array_equal(mine.node_y[:n].view(np.uint32), y[:n].view(np.uint32)), method
    return mine, rep


@needs_ref
@pytest.mark.parametrize("method", ["random", "cluster_fc", "cluster_bc"])
@pytest.mark.parametrize("seed", [1002, 7])
def test_matches_reference_on_generated_designs(method, seed):
    db = generator.small_design(seed)
    mine, rep = compare(db, method, seed=seed)
    n = db.num_movable
    assert np.all(mine.node_x[:n] - mine.node_w[:n] / 2 >= db.core[0] - 1e-3)
    assert np.all(mine.node_y[:n] + mine.node_h[:n] / 2 <= db.core[3] + 1e-3)
    assert np.array_equal(mine.node_x[n:db.num_nodes], db.node_x[n:db.num_nodes])  # fixed nodes stay
    if method != "random":
        assert rep["clusters"] <= max(1, n // 25) * 2 and rep["levels"] > 0


@needs_ref
@pytest.mark.parametrize("method", ["cluster_fc", "cluster_bc"])
def test_cluster_targets_degree_cap_and_disconnected_parts(method):
    db = generator.small_design(3)
    compare(db, method, cluster_target_count=37)
    compare(db, method, ignore_net_degree=3)
    # two disconnected groups and loose nodes: matching stops when nothing is left to merge
    nodes = [(5.0 + i, 5.0, 2.0, 2.0, 0) for i in range(30)] + [(50.0, 50.0, 4.0, 4.0, 1)]
    nets = [[i, i + 1] for i in range(0, 9)] + [[i, i + 1] for i in range(12, 20)] + [[0, 30]]
    small = make_db(nodes, rows=[(float(r), 1.0, 0.0, 1.0, 100) for r in range(100)], nets=nets)
    mine, rep = compare(small, method, cluster_target_count=1)
    assert rep["clusters"] > 1


@needs_ref
def test_wide_nodes_and_random_seed():
    nodes = [(10.0, 10.0, 500.0, 2.0, 0), (10.0, 10.0, 2.0, 500.0, 0), (10.0, 10.0, 3.0, 3.0, 0)]
    db = make_db(nodes, rows=[(float(r), 1.0, 0.0, 1.0, 100) for r in range(100)], nets=[[0, 1, 2]])
    mine, _ = compare(db, "random", seed=11)
    assert mine.node_x[0] == 50.0 and mine.node_y[1] == 50.0  # wider than the core: its centre
    a, _ = compare(db, "random", seed=12)
    assert a.node_x[2] != mine.node_x[2]


def test_unknown_method_is_rejected():
    assert "quadratic" in METHODS
    with pytest.raises(ValueError):
        make_initial_placer("spectral")
