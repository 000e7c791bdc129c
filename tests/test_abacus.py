"""Abacus legalisation (CPU): superplace_b200.legalize against the reference's own legalizeCells
and buildAbacusSegments (src/lg/abacus.cpp, compiled from its sources into oracle/_ref), bit for
bit, on the scenarios of test/test_abacus.cpp (rebuilt here as fixtures) and on seeded random
and generated designs. The scenarios' expected values are asserted directly as well."""
import numpy as np
import pytest

from oracle import ref
from superplace_b200 import generator
from superplace_b200.engine import SpgError
from superplace_b200.legalize import abacus_segments, legalize_cells
from superplace_b200.placedb import F_FILLER, F_FIXED, F_MACRO, F_NI, PlaceDB

needs_ref = pytest.mark.skipif(not ref.available(), reason="oracle/_ref not built")
RESULT_INTS = ("precondition_ok", "cells", "failed", "rows", "segments", "rounded_widths", "selfcheck_overlaps",
               "selfcheck_off_site")


class Fixture:
    """Rows of height 2 at y = 2r (test/test_abacus.cpp:16-21) and nodes added in order, placed
    by their lower-left corner (setLlx/setLly)."""

    def __init__(self, rows=2, sites=20, step=1.0):
        self.rows = [(2.0 * r, 2.0, 0.0, step, sites) for r in range(rows)]
        self.nodes = []
        self.num_movable = 0
        self.fillers = []

    def cell(self, x, y, w=2.0, flags=0, h=2.0):
        f32 = np.float32
        self.nodes.append((float(f32(f32(x) + f32(0.5) * f32(w))), float(f32(f32(y) + f32(0.5) * f32(h))), w, h, flags))
        return len(self.nodes) - 1

    def db(self):
        db = PlaceDB()
        allnodes = self.nodes + self.fillers
        arr = np.array(allnodes, np.float64).reshape(-1, 5)
        db.node_x, db.node_y = arr[:, 0].astype(np.float32), arr[:, 1].astype(np.float32)
        db.node_w, db.node_h = arr[:, 2].astype(np.float32), arr[:, 3].astype(np.float32)
        db.node_flags = arr[:, 4].astype(np.uint8)
        db.num_movable, db.num_nodes, db.num_fillers = self.num_movable, len(self.nodes), len(self.fillers)
        r = np.array(self.rows, np.float64).reshape(-1, 5)
        db.row_ly, db.row_height = r[:, 0].astype(np.float32), r[:, 1].astype(np.float32)
        db.row_lx, db.row_step = r[:, 2].astype(np.float32), r[:, 3].astype(np.float32)
        db.row_num_sites = r[:, 4].astype(np.int32)
        db.compute_regions()
        db.extend_node2pin()
        return db


def llx(db, i):
    return np.float32(db.node_x[i] - np.float32(0.5) * db.node_w[i])


def lly(db, i):
    return np.float32(db.node_y[i] - np.float32(0.5) * db.node_h[i])


def both(db, area=False, reference_trials=False):
    """Ours and the reference's on copies of db: (our db, our result, their x, their y, their result)."""
    mine = db.copy()
    res = legalize_cells(mine, area)
    if not ref.available():
        return mine, res, None, None, None
    r = ref.RefDb(db)
    theirs = ref.abacus(r, area, reference_trials)
    x, y = r.nodes()[:2]
    assert np.array_equal(mine.node_x.view(np.uint32), x.view(np.uint32))
    assert np.array_equal(mine.node_y.view(np.uint32), y.view(np.uint32))
    for k in RESULT_INTS:
        assert res[k] == theirs[k], k
    assert res["disp_mean"] == theirs["disp_mean"] and res["disp_max"] == theirs["disp_max"]
    return mine, res, x, y, theirs


def validate(db):
    """On a row, on its site grid, no two cells overlapping (test/test_abacus.cpp:28-46)."""
    cells = [i for i in range(db.num_movable) if not db.node_flags[i] & (F_MACRO | F_FIXED)]
    for i in cells:
        on_row = False
        for r in range(db.row_ly.shape[0]):
            if abs(lly(db, i) - db.row_ly[r]) < 1e-4:
                site = (llx(db, i) - db.row_lx[r]) / db.row_step[r]
                assert abs(site - round(site)) < 1e-4
                on_row = True
                break
        assert on_row
    for a in cells:
        for b in cells:
            if a < b:
                ox = min(llx(db, a) + db.node_w[a], llx(db, b) + db.node_w[b]) - max(llx(db, a), llx(db, b))
                oy = min(lly(db, a) + db.node_h[a], lly(db, b) + db.node_h[b]) - max(lly(db, a), lly(db, b))
                assert ox <= 1e-4 or oy <= 1e-4


def test_two_cells_split_around_their_target():
    f = Fixture(1)
    f.cell(8, 0), f.cell(8, 0)
    f.num_movable = 2
    db, r, *_ = both(f.db())
    assert r["failed"] == 0 and r["selfcheck_overlaps"] == 0
    assert (llx(db, 0), llx(db, 1)) == (7.0, 9.0)
    validate(db)


def test_segments_around_a_fixed_block():
    f = Fixture(2, 10, 2.0)
    f.cell(8, 0), f.cell(10, 0), f.cell(6.2, 0, 7.6, F_FIXED)
    f.num_movable = 2
    db0 = f.db()
    row, lx, hx = abacus_segments(db0)
    assert list(zip(row, lx, hx)) == [(0, 0.0, 6.0), (0, 14.0, 20.0), (1, 0.0, 20.0)]
    if ref.available():
        rr, rl, rh = ref.abacus_segments(ref.RefDb(db0))
        assert np.array_equal(row, rr) and np.array_equal(lx, rl) and np.array_equal(hx, rh)
    db, r, *_ = both(db0)
    assert r["failed"] == 0 and db.node_x[2] == db0.node_x[2] and db.node_y[2] == db0.node_y[2]
    validate(db)


def test_full_row_spills_to_the_next():
    f = Fixture(3, 2)
    f.cell(0, 2), f.cell(0, 2)
    f.num_movable = 2
    db, r, *_ = both(f.db())
    assert r["failed"] == 0 and lly(db, 0) == 2.0 and lly(db, 1) == 0.0
    validate(db)


def test_off_core_targets_and_rounded_widths():
    f = Fixture(2, 12, 2.0)
    f.cell(-30, -5, 3.0), f.cell(50, 20, 5.0)
    f.num_movable = 2
    db, r, *_ = both(f.db())
    assert r["failed"] == 0 and r["rounded_widths"] == 2
    validate(db)


def test_fixed_ni_and_filler_nodes_stay():
    f = Fixture(2)
    f.cell(4, 0), f.cell(8, 0), f.cell(10, 0, 4.0, F_FIXED, 4.0), f.cell(3, 0, 0.0, F_FIXED | F_NI, 0.0)
    f.num_movable = 2
    f.fillers.append((7.0, 3.0, 2.0, 2.0, F_FILLER))
    db0 = f.db()
    db, r, *_ = both(db0)
    assert r["failed"] == 0
    assert np.array_equal(db.node_x[2:], db0.node_x[2:]) and np.array_equal(db.node_y[2:], db0.node_y[2:])
    validate(db)


def test_overfull_row_leaves_a_failed_cell_in_place():
    f = Fixture(1, 4)
    for _ in range(3):
        f.cell(1, 0)
    f.num_movable = 3
    db, r, *_ = both(f.db())
    assert r["failed"] == 1 and llx(db, 2) == 1.0


def test_unfixed_movable_macro_is_a_no_op():
    f = Fixture()
    f.cell(8, 0), f.cell(8, 0, 4.0, F_MACRO, 4.0)
    f.num_movable = 2
    db0 = f.db()
    db, r, *_ = both(db0)
    assert r["precondition_ok"] == 0
    assert np.array_equal(db.node_x, db0.node_x) and np.array_equal(db.node_y, db0.node_y)


def test_edge_cases_of_the_reference_test():
    f = Fixture(1)
    f.cell(15, 0, 4.0), f.cell(16, 0, 4.0)
    f.num_movable = 2
    db, r, *_ = both(f.db())
    assert r["failed"] == 0
    validate(db)
    f = Fixture(2)  # blocks of different heights cut different rows
    f.cell(2, 0), f.cell(7, 0, 4.0, F_FIXED, 4.0), f.cell(9, 0, 4.0, F_FIXED, 2.0)
    f.num_movable = 1
    row, lx, hx = abacus_segments(f.db())
    assert len(row) == 4 and lx[1] == 13.0 and lx[3] == 11.0
    f = Fixture(0)  # no rows at all
    f.cell(0, 0)
    f.num_movable = 1
    assert both(f.db())[1]["failed"] == 1
    f = Fixture(1)  # a block touching the row from above is no obstacle
    f.cell(15, 0, 2.0), f.cell(3, 2, 10.0, F_FIXED, 2.0)
    f.num_movable = 1
    row, lx, hx = abacus_segments(f.db())
    assert len(row) == 1 and hx[0] == 20.0
    db, r, *_ = both(f.db())
    assert r["failed"] == 0
    f = Fixture(2)  # a fixed macro in the movable segment stays
    f.cell(1, 0, 2.0), f.cell(5, 0, 4.0, F_MACRO | F_FIXED, 4.0)
    f.num_movable = 2
    db0 = f.db()
    db, r, *_ = both(db0)
    assert r["failed"] == 0 and db.node_x[1] == db0.node_x[1] and db.node_y[1] == db0.node_y[1]
    validate(db)


def test_invalid_row_is_rejected_without_moving_anything():
    f = Fixture(1)
    f.cell(2, 0)
    f.num_movable = 1
    db = f.db()
    db.row_step[0] = 0.0
    before = db.node_x.copy()
    with pytest.raises(SpgError, match="invalid site row for Abacus"):
        legalize_cells(db)
    assert np.array_equal(db.node_x, before)
    if ref.available():
        with pytest.raises(ValueError, match="invalid site row for Abacus"):
            ref.abacus(ref.RefDb(db))


def test_area_weight_moves_the_small_cell():
    f = Fixture(1)
    f.cell(10, 0, 4.0), f.cell(10, 0, 2.0)
    f.num_movable = 2
    unit, _, *_ = both(f.db())
    db, r, *_ = both(f.db(), area=True)
    assert llx(unit, 0) == 8.0 and llx(db, 0) == 9.0 and llx(db, 1) == 13.0
    validate(db)


@pytest.mark.parametrize("area", [False, True])
def test_random_rows_match_the_reference_and_its_slow_trials(area):
    """test/test_abacus.cpp:179-205: 40 cells on 5 rows of 80 sites and a fixed block, 100
    seeded trials; the reference's full-state trial path gives the same positions."""
    rng = np.random.default_rng(1234)
    for _ in range(100):
        f = Fixture(5, 80)
        for _ in range(40):
            f.cell(float(int(rng.integers(0, 110)) - 10) + 0.125, float(int(rng.integers(0, 14)) - 3),
                   float(1 + int(rng.integers(0, 5))))
        f.num_movable = 40
        f.cell(30, 2, 10.0, F_FIXED, 4.0)
        db, r, x, y, _ = both(f.db(), area=area)
        assert r["failed"] == 0 and r["selfcheck_overlaps"] == 0 and r["selfcheck_off_site"] == 0
        if ref.available():
            slow = ref.RefDb(f.db())
            ref.abacus(slow, area, reference_trials=True)
            sx, sy = slow.nodes()[:2]
            assert np.array_equal(sx, x) and np.array_equal(sy, y)
        validate(db)


@needs_ref
@pytest.mark.parametrize("seed", [3, 4])
def test_generated_design_matches_the_reference(seed):
    """The 2,000-cell generated design (clustered, overlapping start, fixed pads), as is and
    with two rows cut short and odd site steps."""
    db = generator.small_design(seed)
    both(db)
    db2 = db.copy()
    db2.row_num_sites[5] //= 2
    db2.row_step[7] = np.float32(1.5)
    db2.row_num_sites[7] = int(db2.row_num_sites[7] // 1.5)
    db2.compute_regions()
    mine, r, *_ = both(db2)
    assert r["cells"] > 1900 and r["selfcheck_overlaps"] == 0
