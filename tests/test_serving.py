"""Admission and scheduling of the placement server, on CPU with a stand-in placer: slot and
HBM-budget limits, first-come order, refusal of requests above the budget, and errors
returned to their callers."""
import threading
import time

import numpy as np
import pytest

from superplace_b200 import abi, serving
from superplace_b200.generator import small_design


class Recorder:
    def __init__(self, hold=0.05):
        self.hold = hold
        self.lock = threading.Lock()
        self.running = 0
        self.peak = 0
        self.starts = []

    def __call__(self, req):
        with self.lock:
            self.running += 1
            self.peak = max(self.peak, self.running)
            self.starts.append(req.rid)
        time.sleep(self.hold)
        with self.lock:
            self.running -= 1
        r = abi.Result()
        r.converged = 1
        return r, np.zeros(1, np.float32), np.zeros(1, np.float32)


@pytest.fixture(scope="module")
def db():
    return small_design()


def test_slots_bound_concurrency(db):
    rec = Recorder()
    with serving.PlacementServer(slots=3, placer=rec) as srv:
        futs = [srv.submit(db, 64) for _ in range(9)]
        res = [f.result(timeout=30) for f in futs]
    assert rec.peak == 3 and srv.peak_running == 3
    assert sorted(p.request_id for p in res) == list(range(9))
    assert all(p.t_end >= p.t_start >= p.t_arrival for p in res)


def test_hbm_budget_bounds_concurrency(db):
    need = serving.estimate_device_bytes(db, 64)
    rec = Recorder()
    with serving.PlacementServer(slots=8, hbm_budget_bytes=2.5 * need, placer=rec) as srv:
        for f in [srv.submit(db, 64) for _ in range(6)]:
            f.result(timeout=30)
    assert rec.peak == 2 and srv.peak_bytes <= 2.5 * need


def test_first_come_first_served(db):
    rec = Recorder(hold=0.01)
    with serving.PlacementServer(slots=1, placer=rec) as srv:
        for f in [srv.submit(db, 64) for _ in range(5)]:
            f.result(timeout=30)
    assert rec.starts == list(range(5))


def test_request_above_budget_is_refused(db):
    with serving.PlacementServer(slots=2, hbm_budget_bytes=1e6, placer=Recorder()) as srv:
        with pytest.raises(ValueError):
            srv.submit(db, 64)


def test_errors_reach_the_caller(db):
    rec = Recorder(hold=0.01)

    def place(req):
        if req.rid == 0:
            raise RuntimeError("placement failed")
        return rec(req)

    with serving.PlacementServer(slots=1, placer=place) as srv:
        f = srv.submit(db, 64)
        with pytest.raises(RuntimeError):
            f.result(timeout=30)
        # the failed request released its slot and budget: the next one runs
        assert srv.submit(db, 64).result(timeout=30).result.converged == 1


def test_precision_choice():
    assert serving.choose_precision(64, "auto") == abi.POISSON_FP32
    assert serving.choose_precision(256, "auto") == abi.POISSON_BF16X3
    assert serving.choose_precision(256, "fp32") == abi.POISSON_FP32


def test_poisson_arrivals_rate():
    a = serving.poisson_arrivals(50.0, 2000, seed=3)
    assert np.all(np.diff(a) > 0)
    assert abs(len(a) / a[-1] - 50.0) < 5.0
