"""The fillers' spatial reorder at the loop's pause (GPU only).

At the reorder iteration the stage loop pauses and permutes the filler segment of the opt set
by bin tile of the current positions (filler_order.cu): every optimizer vector the loop still
reads, the snapshots and the fillers' node ids. It changes no value, only the order of the FP64
sums over the opt set. Checked on a 20k-cell design with its fillers (above the 4096-filler
threshold; the 2k-cell tests never reorder):

  * the graph loop and the host-driven loop give the same stage bit for bit, and two runs
    give the same stage (the permutation is deterministic);
  * against the same stage without the reorder (SPG_FILLER_ORDER=0, run in a child process
    because the switch is read once per process): the same iteration count within 2, the final
    HPWL within 1e-4 and the overflow within 1e-3;
  * every node ends inside the core and the fixed nodes do not move (the node ids moved with
    their values).
"""
import json
import os
import subprocess
import sys

import numpy as np
import pytest

from superplace_b200 import abi, engine, generator

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

CHILD = r"""
import json, sys
sys.path.insert(0, {root!r})
from superplace_b200 import abi, engine, generator
db, grid = generator.scaled_design(7, 20000)
engine.initialize_fillers(db, 1.0, 1002)
r = engine.EPlace(db, abi.default_params(gp_bin_dim=grid)).run(abi.STAGE_MGP)
print(json.dumps({{"iterations": r.iterations, "hpwl": r.hpwl, "overflow": r.overflow}}))
"""


def design():
    db, grid = generator.scaled_design(7, 20000)
    engine.initialize_fillers(db, 1.0, 1002)
    return db, grid


def run(host_loop=False, monkeypatch=None):
    if monkeypatch is not None:
        if host_loop:
            monkeypatch.setenv("SPG_HOST_LOOP", "1")
        else:
            monkeypatch.delenv("SPG_HOST_LOOP", raising=False)
    db, grid = design()
    x0 = db.node_x.copy()
    r = engine.EPlace(db, abi.default_params(gp_bin_dim=grid)).run(abi.STAGE_MGP)
    return db, x0, r


def test_design_is_above_the_reorder_threshold():
    db, _ = design()
    assert db.num_fillers >= 4096


def test_reorder_graph_loop_matches_host_loop(monkeypatch):
    dg, _, rg = run(False, monkeypatch)
    dh, _, rh = run(True, monkeypatch)
    assert rg.iterations > 8  # the loop passed the reorder pause
    assert (rg.iterations, rg.hpwl, rg.overflow) == (rh.iterations, rh.hpwl, rh.overflow)
    assert np.array_equal(dg.node_x, dh.node_x) and np.array_equal(dg.node_y, dh.node_y)
    d2, _, r2 = run(False, monkeypatch)
    assert (r2.iterations, r2.hpwl) == (rg.iterations, rg.hpwl)
    assert np.array_equal(d2.node_x, dg.node_x) and np.array_equal(d2.node_y, dg.node_y)


def test_reorder_changes_only_the_sum_order(monkeypatch):
    db, x0, r = run(False, monkeypatch)
    env = dict(os.environ, SPG_FILLER_ORDER="0")
    env.pop("SPG_HOST_LOOP", None)
    out = subprocess.run([sys.executable, "-c", CHILD.format(root=ROOT)], env=env, capture_output=True, text=True,
                         timeout=600, check=True)
    plain = json.loads(out.stdout.strip().splitlines()[-1])
    assert abs(r.iterations - plain["iterations"]) <= 2, (r.iterations, plain)
    assert abs(r.hpwl - plain["hpwl"]) <= 1e-4 * plain["hpwl"], (r.hpwl, plain)
    assert abs(r.overflow - plain["overflow"]) <= 1e-3, (r.overflow, plain)
    lx, ly, hx, hy = db.core
    n = db.total_nodes
    assert np.all(db.node_x[:n] >= lx - 1e-3) and np.all(db.node_x[:n] <= hx + 1e-3)
    assert np.all(db.node_y[:n] >= ly - 1e-3) and np.all(db.node_y[:n] <= hy + 1e-3)
    fixed = (db.node_flags & abi.F_FIXED) != 0
    assert np.array_equal(db.node_x[: db.num_nodes][fixed[: db.num_nodes]], x0[: db.num_nodes][fixed[: db.num_nodes]])
