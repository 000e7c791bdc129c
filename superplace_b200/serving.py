"""Placement serving on one GPU: continuous batching of independent global-placement requests.

A request is one placement instance (a PlaceDB with its fillers) and a bin grid; its result
is the converged mGP placement (EPlace::run(kMGP), src/gp/eplace.cpp:356-515). The server
keeps up to `slots` requests on the device at once:

* admission: requests wait in arrival order; the oldest is admitted when a slot is free and
  its estimated device footprint fits the HBM budget beside the requests already running;
* each slot owns a GpContext (its own streams, pinned staging memory, device buffers from the
  library's stream-ordered pool, and its own loop graph) kept across requests: a new request
  is loaded into it (spg_ctx_load), reusing what fits, and runs on the slot's worker thread,
  so the kernels of all running requests overlap on the device;
* every result is the same as the request's result alone: a context's work depends only on
  its own inputs, and every reduction in the engine has a fixed order.

`PlacementServer(slots=1, precision="fp32")` is the one-at-a-time plain-FP32 baseline.
Each slot's context uses two CUDA streams; a serving process with many slots should set
CUDA_DEVICE_MAX_CONNECTIONS to twice the slot count before CUDA starts (bench.py --serve does),
so that the slots' streams do not share hardware work queues.
"""
from __future__ import annotations

import collections
import threading
import time
from concurrent.futures import Future
from dataclasses import dataclass, field

import numpy as np

from . import abi
from .placedb import PlaceDB


def estimate_device_bytes(db: PlaceDB, bin_dim: int) -> int:
    """A conservative device footprint of one placement context (bytes): node, pin and net
    arrays, the optimizer pool (18 vectors of 2 floats per optimised node), bin maps and the
    Poisson plan (bases, work and split planes), plus a fixed allowance for streams, graphs
    and pool granularity."""
    total = int(db.num_nodes) + int(db.num_fillers)
    pins, nets, bins = int(db.num_pins), int(db.num_nets), int(bin_dim) ** 2
    return (48 * total + 40 * pins + 12 * nets + 216 * total + 200 * bins + (64 << 20))


def choose_precision(bin_dim: int, precision: str) -> int:
    if precision == "fp32":
        return abi.POISSON_FP32
    if precision == "bf16x3":
        return abi.POISSON_BF16X3
    # auto: the tensor-core form where the grid tiles by 128, else plain FP32
    return abi.POISSON_BF16X3 if bin_dim % 128 == 0 else abi.POISSON_FP32


@dataclass
class Placement:
    """The result of one request: the mGP result, the placed positions and its timeline
    (perf_counter seconds)."""
    request_id: int
    result: abi.Result
    x: np.ndarray
    y: np.ndarray
    t_arrival: float
    t_start: float
    t_end: float
    device_bytes: int
    phases_ms: dict = field(default_factory=dict)  # host time per phase, when the placer reports it

    @property
    def latency(self) -> float:
        return self.t_end - self.t_arrival


@dataclass
class _Request:
    rid: int
    db: PlaceDB
    bin_dim: int
    precision: int
    t_arrival: float
    need: int
    future: Future = field(default_factory=Future)


class _Slot:
    """The device state of one slot: a placement context kept across requests and reloaded
    with each new netlist (spg_ctx_load), so its streams, staging memory, device buffers and
    loop graph are reused instead of being built and torn down per request."""

    def __init__(self):
        self.ctx = None

    def place(self, req: _Request):
        from . import engine

        t = [time.perf_counter()]
        # the slots' solves run side by side on the device: separate launches (no grid barriers)
        params = abi.default_params(gp_bin_dim=req.bin_dim, poisson_precision=req.precision,
                                    poisson_single_launch=0)
        if self.ctx is None:
            self.ctx = engine.GpContext(req.db, params)
        else:
            self.ctx.load(req.db, params)
        ctx = self.ctx
        t.append(time.perf_counter())
        ctx.set_positions(req.db.node_x, req.db.node_y)
        ctx.set_flags(req.db.node_flags)
        t.append(time.perf_counter())
        r = ctx.run(abi.STAGE_MGP)
        t.append(time.perf_counter())
        x, y = ctx.positions()
        t.append(time.perf_counter())
        names = ("load", "h2d", "stage_run", "d2h")
        phases = {k: (b - a) * 1e3 for k, a, b in zip(names, t[:-1], t[1:])}
        phases["device_loop"] = r.elapsed_ms
        return r, x, y, phases

    def close(self):
        if self.ctx is not None:
            self.ctx.close()
            self.ctx = None


def _place_on_device(req: _Request, slot: _Slot | None = None):
    """Place one request on the device (in the slot's context when one is given)."""
    own = slot is None
    slot = slot or _Slot()
    try:
        return slot.place(req)
    finally:
        if own:
            slot.close()


class PlacementServer:
    """Continuous-batching placement service (see the module docstring).

    placer: the function that places one request (the device engine by default; tests of the
    admission logic pass a stand-in)."""

    def __init__(self, slots: int = 8, hbm_budget_bytes: float = 150e9, precision: str = "auto",
                 placer=_place_on_device):
        if slots < 1:
            raise ValueError("slots must be >= 1")
        self.slots = slots
        self.budget = int(hbm_budget_bytes)
        self.precision = precision
        self._placer = placer
        self._cv = threading.Condition()
        self._queue: collections.deque[_Request] = collections.deque()
        self._in_use = 0
        self._running = 0
        self._closed = False
        self._next_id = 0
        self.peak_running = 0
        self.peak_bytes = 0
        self._workers = [threading.Thread(target=self._work, daemon=True, name=f"placement-slot-{i}")
                         for i in range(slots)]
        for t in self._workers:
            t.start()

    def submit(self, db: PlaceDB, bin_dim: int, t_arrival: float | None = None) -> Future:
        """Queue one placement; the Future resolves to a Placement (or raises the engine's
        SpgError). Requests larger than the whole budget are refused at once."""
        need = estimate_device_bytes(db, bin_dim)
        if need > self.budget:
            raise ValueError(f"request needs ~{need / 1e9:.1f} GB, above the {self.budget / 1e9:.1f} GB budget")
        with self._cv:
            if self._closed:
                raise RuntimeError("server is closed")
            req = _Request(self._next_id, db, int(bin_dim), choose_precision(bin_dim, self.precision),
                           time.perf_counter() if t_arrival is None else t_arrival, need)
            self._next_id += 1
            self._queue.append(req)
            self._cv.notify_all()
        return req.future

    def close(self):
        with self._cv:
            self._closed = True
            self._cv.notify_all()
        for t in self._workers:
            t.join()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def _admit(self) -> _Request | None:
        """The oldest request, once it fits the budget beside the running ones (FIFO: a big
        request at the head is not overtaken)."""
        with self._cv:
            while True:
                if self._queue and self._in_use + self._queue[0].need <= self.budget:
                    req = self._queue.popleft()
                    self._in_use += req.need
                    self._running += 1
                    self.peak_running = max(self.peak_running, self._running)
                    self.peak_bytes = max(self.peak_bytes, self._in_use)
                    return req
                if self._closed and not self._queue:
                    return None
                self._cv.wait()

    def _release(self, req: _Request):
        with self._cv:
            self._in_use -= req.need
            self._running -= 1
            self._cv.notify_all()

    def _work(self):
        slot = _Slot()
        try:
            self._serve(slot)
        finally:
            slot.close()

    def _serve(self, slot: _Slot):
        while True:
            req = self._admit()
            if req is None:
                return
            t0 = time.perf_counter()
            try:
                got = self._placer(req, slot) if self._placer is _place_on_device else self._placer(req)
                r, x, y = got[:3]
                out = Placement(req.rid, r, x, y, req.t_arrival, t0, time.perf_counter(), req.need,
                                got[3] if len(got) > 3 else {})
                req.future.set_result(out)
            except BaseException as e:  # the request's error goes to its caller
                req.future.set_exception(e)
            finally:
                self._release(req)


def poisson_arrivals(rate: float, n: int, seed: int = 7) -> np.ndarray:
    """Arrival offsets (seconds) of n requests of a Poisson process at `rate` per second."""
    rng = np.random.default_rng(seed)
    return np.cumsum(rng.exponential(1.0 / rate, n))


def replay(server: PlacementServer, requests, arrivals) -> list[Placement]:
    """Submit (db, bin_dim) requests at their arrival offsets (real time) and wait for all."""
    t0 = time.perf_counter()
    futs = []
    for (db, dim), a in zip(requests, arrivals):
        now = time.perf_counter() - t0
        if a > now:
            time.sleep(a - now)
        futs.append(server.submit(db, dim, t_arrival=t0 + a))
    return [f.result() for f in futs]


def summarize(results: list[Placement]) -> dict:
    lat = np.array([r.latency for r in results])
    t_first = min(r.t_arrival for r in results)
    t_last = max(r.t_end for r in results)
    phases = {}
    for k in ("load", "h2d", "stage_run", "d2h", "device_loop"):
        v = [r.phases_ms[k] for r in results if k in r.phases_ms]
        if v:
            phases[k] = float(np.mean(v))
    return {"requests": len(results), "placements_per_s": len(results) / (t_last - t_first),
            "mean_phase_ms": phases,
            "p50_ms": float(np.percentile(lat, 50) * 1e3), "p99_ms": float(np.percentile(lat, 99) * 1e3),
            "mean_ms": float(lat.mean() * 1e3),
            "converged": int(sum(int(r.result.converged) for r in results))}
