"""The GP stage sequence on a mixed-size design (GPU only), against the reference's own run.

GlobalPlaceStage::run (src/stages/gp_stage.cpp:99-215) places mGP, legalises the macros (host
SA, not part of this path), freezes them, re-scatters the fillers with seed offset 1, runs
FILLERONLY for a fixed number of iterations, then cGP. Each stage here starts the device and
the reference build (oracle/_ref) from the same positions and flags:

  * mGP with 10 movable macros (footprints above 16 bins: the block-per-node density and gather
    kernels): converges like the reference (iterations within 25%, HPWL within 2%);
  * FILLERONLY: exactly filler_only_iters iterations, and only fillers move (every cell and
    macro keeps its position bit for bit), as in the reference;
  * cGP with the macros frozen: converges below the cGP target like the reference, and no
    macro moves (test/test_eplace.cpp:444-477, gp_stage.cpp:205-215).
"""
import numpy as np
import pytest

from superplace_b200 import abi, engine, generator
from superplace_b200.placedb import F_FIXED, F_MACRO

pytestmark = pytest.mark.gpu

BINS = 64


def mixed_small(seed=1002):
    rng = np.random.default_rng(seed + 17)
    w = rng.integers(2, 17, 2000).astype(np.float32)
    db = generator.build_design(seed=seed, die=600.0, row_h=12.0, n_cells=2000, cell_w=w, n_nets=2100,
                                n_movable_macros=10, movable_macro_frac=0.2, movable_macro_rows=(3, 8),
                                n_pads=64, name="mixed_2k")
    engine.initialize_fillers(db, 1.0, seed)
    return db


def params():
    return abi.default_params(gp_bin_dim=BINS)


def run_both(db, stage):
    """The stage on the device and on the reference build, from the same db state."""
    from oracle import ref

    if not ref.available():
        pytest.skip("oracle/_ref/libspref.so not built")
    dev = db.copy()
    r = engine.EPlace(dev, params()).run(stage)
    rdb = ref.RefDb(db)
    res, rows = rdb.eplace(params(), stage=stage)
    x, y = rdb.nodes()[:2]
    return dev, r, res, rows, x, y


@pytest.fixture(scope="module")
def after_mgp():
    db = mixed_small()
    assert np.count_nonzero(db.node_flags[: db.num_movable] & F_MACRO) == 10
    dev, r, res, _, _, _ = run_both(db, abi.STAGE_MGP)
    return db, dev, r, res


def test_mixed_mgp_converges_like_reference(after_mgp):
    _, _, r, res = after_mgp
    assert r.converged == 1 and r.overflow < 0.10
    assert abs(r.iterations - res["iterations"]) <= 0.25 * res["iterations"]
    assert abs(r.hpwl - res["hpwl"]) <= 0.02 * res["hpwl"]


@pytest.fixture(scope="module")
def frozen(after_mgp):
    """mGP result with the macros frozen and the fillers re-scattered (gp_stage.cpp:168-186)."""
    _, dev, _, _ = after_mgp
    db = dev.copy()
    m = (db.node_flags[: db.num_movable] & F_MACRO) != 0
    db.node_flags[: db.num_movable][m] |= F_FIXED
    engine.scatter_fillers(db, 1002, seed_offset=1)
    return db


def test_filler_only_moves_only_fillers(frozen):
    db = frozen
    dev, r, res, _, rx, ry = run_both(db, abi.STAGE_FILLER_ONLY)
    iters = abi.default_params().filler_only_iters
    assert r.iterations == iters and res["iterations"] == iters
    real = slice(0, db.num_nodes)
    assert np.array_equal(dev.node_x[real], db.node_x[real]) and np.array_equal(dev.node_y[real], db.node_y[real])
    assert np.array_equal(rx[real], db.node_x[real]) and np.array_equal(ry[real], db.node_y[real])
    fill = slice(db.num_nodes, db.num_nodes + db.num_fillers)
    assert not np.array_equal(dev.node_x[fill], db.node_x[fill])
    # the HPWL of the real nodes does not change, and both runs report it alike
    assert abs(r.hpwl - res["hpwl"]) <= 1e-9 * res["hpwl"]


def test_cgp_keeps_macros_frozen_and_converges(frozen):
    db = frozen.copy()
    engine.EPlace(db, params()).run(abi.STAGE_FILLER_ONLY)
    dev, r, res, _, _, _ = run_both(db, abi.STAGE_CGP)
    macros = np.nonzero(db.node_flags[: db.num_movable] & F_MACRO)[0]
    assert np.array_equal(dev.node_x[macros], db.node_x[macros])
    assert np.array_equal(dev.node_y[macros], db.node_y[macros])
    target = abi.default_params().cgp_target_overflow
    assert r.converged == 1 and r.overflow < target
    assert res["converged"] == 1
    assert abs(r.iterations - res["iterations"]) <= 0.25 * res["iterations"] + 2
    assert abs(r.hpwl - res["hpwl"]) <= 0.02 * res["hpwl"]
