import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs an sm_100 (B200) device")


def load_golden(name):
    return dict(np.load(os.path.join(GOLDEN, name)))


def golden_small_db(with_fillers=True):
    """The 2,000-cell design stored in tests/golden/small_design.npz (inputs of the
    reference run), optionally with the reference's fillers."""
    from superplace_b200.placedb import PlaceDB

    g = load_golden("small_design.npz")
    db = PlaceDB()
    for k in ("node_x", "node_y", "node_w", "node_h", "node_flags", "pin_offset_x",
              "pin_offset_y", "pin2node", "pin2net", "net2pin_start", "flat_net2pin",
              "node2pin_start", "flat_node2pin", "row_ly", "row_height", "row_lx", "row_step",
              "row_num_sites"):
        setattr(db, k, g["in_" + k].copy())
    db.num_movable, db.num_nodes, db.num_fillers = (int(v) for v in g["in_counts"])
    db.core = tuple(float(v) for v in g["in_core"])
    db.row_height_mode = float(g["in_row_height_mode"])
    db.total_row_area = float(g["in_total_row_area"])
    db.name = "small_2k"
    if with_fillers:
        info = g["filler_info"]
        db.set_fillers(int(info[0]), float(info[1]), float(info[2]), g["filler_x"], g["filler_y"])
    return db, g


@pytest.fixture(scope="session")
def small():
    return golden_small_db(True)
