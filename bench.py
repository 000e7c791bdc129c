"""Benchmark: mGP iterations/s on the 211k-cell synthetic netlist (512x512 bins, tau 0.10).

One "step" is one complete mGP stage (lambda_0 probe, initial-step estimate, Nesterov
iterations with backtracking until tau < 0.10 or stagnation) from the same initial
placement. Metric: mGP iterations per second = sum(iterations) / sum(iteration-loop time),
the reference's own definition (mGP_iterations / durations_ms["mGP"],
src/gp/eplace.cpp:310,515).

  value  loop time from CUDA events on the engine's stream (inputs resident in HBM)
  e2e    the same metric through the public API (EPlace.run on a host PlaceDB whose positions
         and flags sit in page-locked memory): H2D of positions/flags, stage set-up, the loop
         and the D2H of the delivered positions, bracketed by CUDA events on the engine's
         stream

Usage: python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                       [--precision bf16x3|fp32] [--workload large|small]
       python bench.py --poisson-sweep | --precision-study | --mixed-study | --serve | --bookshelf | --qp
                       | --flow
                                                                    (studies: JSON lines of their own)
The default Poisson arithmetic is split-BF16 on tcgen05 (bf16x3); fp32 is the plain FP32 form.
Multi-GPU: replicas only (each rank places its own copy; "scaling": "weak").
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

from superplace_b200 import abi, generator  # noqa: E402

WORKLOADS = {
    "large": dict(desc="mGP to tau<0.10, 211k-cell synthetic netlist (543 fixed macros, 35% "
                       "blocked), 221k nets, 512x512 bins", bin_dim=512),
    "small": dict(desc="mGP to tau<0.10, 2k-cell synthetic netlist, 64x64 bins", bin_dim=64),
}
METRIC = "mGP iters/s at 211k cells (tau=0.10)"


def make_design(workload, seed=1002):
    if workload == "large":
        return generator.large_design(seed)
    return generator.small_design(seed)


def dist_env():
    rank = int(os.environ.get("RANK", 0))
    world = int(os.environ.get("WORLD_SIZE", 1))
    local = int(os.environ.get("LOCAL_RANK", 0))
    return rank, world, local


def max_over_ranks(values, world, device):
    """The elementwise maximum of per-rank times over the job's ranks (one all-reduce on the
    job's process group, on `device`); the values themselves when the job has one rank."""
    if world <= 1:
        return [float(v) for v in values]
    import torch
    import torch.distributed as dist

    t = torch.tensor([float(v) for v in values], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return [float(v) for v in t.tolist()]


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.idx = gpu_index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "100", "-i", str(self.idx)], stdout=subprocess.PIPE,
                stderr=subprocess.DEVNULL, text=True)
            self.th = threading.Thread(target=self._read, daemon=True)
            self.th.start()
        except (OSError, FileNotFoundError):
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for n, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return p["hbm_gbs"], p["bf16_tflops"], "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, 1590.0, "fallback"


# ------------------------------------------------------------------ reference arm
def ref_fillers(db, ref):
    """The reference's own initializeFillers (src/gp/filler.cpp:47-139) on a copy of db, its
    fillers appended to db (no library of this package is loaded)."""
    r = ref.RefDb(db)
    info = r.fillers_init(1.0, 1002)
    x, y, _, _, _ = r.nodes()
    db.set_fillers(int(info[0]), info[1], info[2], x[db.num_nodes:], y[db.num_nodes:])


def run_reference(args):
    rank, world, _ = dist_env()
    if rank != 0:
        return 0
    from oracle import ref

    if not ref.available():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libspref.so not built"}))
        return 0
    db = make_design(args.workload)
    ref_fillers(db, ref)
    threads = os.cpu_count() or 1
    ref.lib().spref_set_threads(threads)
    sample_iters = args.ref_iters
    params = abi.default_params(gp_bin_dim=WORKLOADS[args.workload]["bin_dim"],
                                gp_max_iter=sample_iters if sample_iters > 0 else 2000)
    # the CPU run needs no warm-up: one untimed stage at most, so the arm ends in minutes
    iters, ms = [], []
    for k in range(min(args.warmup, 1) + args.steps):
        r = ref.RefDb(db)
        res, rows = r.eplace(params)
        if k >= min(args.warmup, 1):
            iters.append(int(res["iterations"]))
            ms.append(res["elapsed_ms"])
    value = sum(iters) / (sum(ms) / 1e3)
    what = (f"first {sample_iters} mGP iterations" if sample_iters > 0 else
            "full mGP stages (lambda_0 probe, initial step, iterations to tau<0.10)")
    sample = (f"{what} of the same instance, each from the same start, on the reference's CPU "
              f"EPlace built from its sources (FFT stand-in for FFTW), {threads} threads")
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "iter/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": min(args.warmup, 1),
        "ms_per_step": sum(ms) / len(ms), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": WORKLOADS[args.workload]["desc"], "cells": int(db.num_movable),
                   "fillers": int(db.num_fillers), "pins": int(db.num_pins),
                   "nets": int(db.num_nets), "bins": WORKLOADS[args.workload]["bin_dim"],
                   "step": "one full mGP stage run" if sample_iters <= 0 else f"{sample_iters}-iteration sample",
                   "iterations_per_step": iters},
        "cpu_baseline": {"value": value, "unit": "iter/s", "cores": threads, "kind": "reference",
                         "sample": sample},
        "e2e": {"value": value, "unit": "iter/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))
    return 0


# ------------------------------------------------------------------ our arm
def cpu_baseline_sample(db, workload):
    """The reference's CPU EPlace on the same instance: one full mGP stage (the same work as
    one step of this arm), all host cores."""
    try:
        from oracle import ref

        if not ref.available():
            return None
        threads = os.cpu_count() or 1
        ref.lib().spref_set_threads(threads)
        r = ref.RefDb(db)
        res, _ = r.eplace(abi.default_params(gp_bin_dim=WORKLOADS[workload]["bin_dim"]))
        v = res["iterations"] / (res["elapsed_ms"] / 1e3)
        return {"value": v, "unit": "iter/s", "cores": threads, "kind": "reference",
                "sample": f"one full mGP stage ({int(res['iterations'])} iterations, "
                          f"{res['elapsed_ms'] / 1e3:.1f} s) of this instance on the reference's CPU "
                          f"EPlace built from its sources (FFT stand-in for FFTW)"}
    except Exception as e:  # the baseline must not hide our number
        return {"value": None, "unit": "iter/s", "cores": 0, "kind": "reference",
                "sample": f"failed: {e}"}


def fp32_arm(db, workload, init_x, init_y, steps):
    """The plain FP32 GPU form (FP32 SIMT cosine contractions) on the same instance and start,
    timed the same way as the headline arm: mGP iterations per second of loop time."""
    from superplace_b200 import engine

    params = abi.default_params(gp_bin_dim=WORKLOADS[workload]["bin_dim"], poisson_precision=abi.POISSON_FP32)
    ep = engine.EPlace(db, params)
    iters, ms = [], []
    for k in range(1 + steps):
        db.node_x[:] = init_x
        db.node_y[:] = init_y
        r = ep.run(abi.STAGE_MGP)
        if k:
            iters.append(r.iterations)
            ms.append(r.elapsed_ms)
    ep.ctx.close()
    return sum(iters) / (sum(ms) / 1e3), iters


# DRAM bytes per launch (dram__bytes_read.sum + dram__bytes_write.sum) of each part, from ncu
# captures of the 211k-cell workload with the split-BF16 Poisson (caches flushed before each
# replayed launch, so these are cold-L2 figures; writes that stay in L2 at the end of a launch
# are not counted). The Poisson part is its five launches of one solve (its first operand comes
# from the rho kernel); the WA part is the nets pass and the cells' pass 2.
PROFILED_DRAM_BYTES = {
    ("large", "bf16x3"): {"update": 40.17e6, "wa": 25.76e6, "rho": 6.31e6, "poisson": 13.77e6,
                          "assemble": 39.18e6,
                          "source": "profiles/mgp_211k_bf16x3_kernels.md"},
}


def part_rooflines(parts, db, dim, hbm_gbs, bf16_tflops, precision, traffic=None):
    """Algorithmic bytes (or flops) of each iteration part per launch, divided by its
    warm-L2 device time. Bytes count every array the part must touch once (FP32/int32);
    fillers share their attributes as launch constants, so only cells read per-node ones:
      update     40 B per optimised node (u, v, g in; v', u' out) + 60 B per cell (x, y into
                 the node arrays; meta, geometry, clamp box, node index) + 16 B per bin (the
                 two fixed-point maps it scatters into)
      wa         32 B per pin + 8 B per net (pass 1: pin ids, offsets, positions in; 2 terms
                 out) + 8 B per pin + 24 B per cell (pass 2: terms and meta in; 2 sums out)
      scatter    25 B per density node outside the opt set + 16 B per bin (only FILLERONLY
                 and cGP have such nodes)
      rho        44 B per bin (maps, terminal, base in; rho out; maps cleared)
      poisson    14 M^3 flops (16 B per bin of I/O)
      assemble   32 B per optimised node (u, uPrev, gPrevTmp in; g out) + 48 B per cell
                 (meta, geometry, area, the WA pass-2 sums) + 8 B per bin (the field maps it
                 gathers from)
    traffic: measured DRAM bytes per launch by part (PROFILED_DRAM_BYTES), when known.
    """
    n_opt = db.num_movable + db.num_fillers
    cells = db.num_movable
    n_dens = n_opt
    pins, nets, bins = db.num_pins, db.num_nets, dim * dim
    by = {"update": 40 * n_opt + 60 * cells + 16 * bins, "wa": 40 * pins + 8 * nets + 24 * cells,
          "scatter": 25 * n_dens + 16 * bins, "rho": 44 * bins,
          "assemble": 32 * n_opt + 48 * cells + 8 * bins}
    traffic = traffic or {}
    out = {}
    for k, us in parts.items():
        if k == "poisson":
            ach = 14.0 * dim ** 3 / (us * 1e-6) / 1e12
            out[k] = {"us": us, "bound": "tensor", "achieved": ach, "peak": bf16_tflops,
                      "unit": "TFLOP/s", "frac": ach / bf16_tflops,
                      "note": "algorithmic flops; split-BF16 executes 3x" if precision else
                              "FP32 SIMT path, measured against the bf16 tensor peak"}
        elif k in by:
            ach = by[k] / (us * 1e-6) / 1e9
            out[k] = {"us": us, "bound": "hbm", "achieved": ach, "peak": hbm_gbs, "unit": "GB/s",
                      "frac": ach / hbm_gbs, "bytes": by[k]}
        else:
            out[k] = {"us": us}
        out[k]["traffic"] = traffic.get(k)
    return out


def time_poisson(dim, step_x, step_y, precision, reps=50):
    """Average device time of one Poisson solve (the dominant kernel group) with CUDA
    events on the launching stream; inputs resident."""
    import torch

    from superplace_b200 import engine

    be = engine.PoissonBackend(dim, dim, step_x, step_y, precision)
    rng = np.random.default_rng(7)
    rho = torch.from_numpy(rng.random((dim, dim), dtype=np.float32)).cuda()
    out = [torch.empty_like(rho) for _ in range(3)]
    s = torch.cuda.current_stream()
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device="cuda")  # 256 MB > L2
    for _ in range(5):
        be.solve_device(rho.data_ptr(), *(o.data_ptr() for o in out), stream=s.cuda_stream)
    times = []
    for _ in range(reps):
        flush.zero_()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(s)
        be.solve_device(rho.data_ptr(), *(o.data_ptr() for o in out), stream=s.cuda_stream)
        e1.record(s)
        e1.synchronize()
        times.append(e0.elapsed_time(e1))
    return statistics.median(times)


def run_ours(args):
    import torch
    import torch.distributed as dist

    from superplace_b200 import engine

    rank, world, local = dist_env()
    if world > 1:
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=600))
    torch.cuda.set_device(local)
    precision = abi.POISSON_BF16X3 if args.precision == "bf16x3" else abi.POISSON_FP32
    db = make_design(args.workload)
    engine.initialize_fillers(db, 1.0, 1002)
    engine.pin_positions(db)  # the step's inputs and result in page-locked host memory
    init_x, init_y = db.node_x.copy(), db.node_y.copy()
    params = abi.default_params(gp_bin_dim=WORKLOADS[args.workload]["bin_dim"],
                                poisson_precision=precision)
    ep = engine.EPlace(db, params)
    stream = torch.cuda.ExternalStream(ep.ctx.stream())

    def reset():  # every step places the same instance from the same start (not timed)
        db.node_x[:] = init_x
        db.node_y[:] = init_y

    def step():
        return ep.run(abi.STAGE_MGP)

    for _ in range(args.warmup):
        reset()
        step()
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    launches0 = engine.launch_count()
    iters, loop_ms, e2e_ms, hpwl, tau = [], [], [], [], []
    with ClockSampler(local) as clk:
        for _ in range(args.steps):
            reset()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            r = step()
            e1.record(stream)
            e1.synchronize()
            e2e_ms.append(e0.elapsed_time(e1))
            iters.append(r.iterations)
            loop_ms.append(r.elapsed_ms)
            hpwl.append(r.hpwl)
            tau.append(r.overflow)
    torch.cuda.synchronize()
    launches = engine.launch_count() - launches0
    if world > 1:
        dist.barrier()
    t_loop = sum(loop_ms) / 1e3
    t_e2e = sum(e2e_ms) / 1e3
    t_loop, t_e2e = max_over_ranks([t_loop, t_e2e], world, "cuda")
    total_iters = sum(iters) * world
    value = total_iters / t_loop
    e2e = total_iters / t_e2e
    if rank == 0:
        info = ep.ctx.grid_info()
        dim = info["dim"]
        hbm, bf16, peak_kind = peaks()
        parts = ep.ctx.profile(reps=20)
        traffic = PROFILED_DRAM_BYTES.get((args.workload, args.precision), {})
        kern = part_rooflines(parts, db, dim, hbm, bf16, precision, traffic)
        # the dominant kernel: the longest part of the iteration's critical chain (WA runs on the
        # side stream beside the fillers' step, so it is listed under `kernels` but not chosen)
        dom = max((k for k in kern if k not in ("evaluation", "wa")), key=lambda k: kern[k]["us"])
        d = kern[dom]
        total = db.total_nodes
        h2d = 2 * 4 * total + total  # positions x, y and flags
        d2h = 2 * 4 * total
        line = {
            "metric": METRIC, "value": value, "unit": "iter/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": sum(loop_ms) / len(loop_ms), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None,
            "dtype": "f32" if precision == abi.POISSON_FP32 else "bf16x3+f32",
            "data": "synthetic",
            "config": {"workload": WORKLOADS[args.workload]["desc"], "cells": int(db.num_movable),
                       "fillers": int(db.num_fillers), "pins": int(db.num_pins),
                       "nets": int(db.num_nets), "bins": dim,
                       "poisson": args.precision, "step": "one full mGP stage run",
                       "loop": "conditional CUDA graph" if ep.ctx.graph_loop() else "host-driven",
                       "iterations_per_step": iters, "final_hpwl": hpwl, "final_tau": tau,
                       "l2": "no flush between iterations: the per-iteration working set "
                             "(~160 MB) exceeds the 126 MB L2; part timings are warm-L2 as "
                             "inside the loop",
                       "parallelism": f"replicas x{world}"},
            "e2e": {"value": e2e, "unit": "iter/s", "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h},
            "gpu_launches": launches,
            "roofline": {"bound": d["bound"], "achieved": d["achieved"], "peak": d["peak"],
                         "unit": d["unit"], "frac": d["frac"], "traffic": d["traffic"],
                         "traffic_source": traffic.get("source"),
                         "kernel": dom, "us_per_launch": d["us"], "peak_kind": peak_kind},
            "kernels": kern,
            "clocks": clk.summary(),
        }
        # the FP32 arm, the serving leg and the CPU baseline are one-GPU records: a job of
        # several ranks reports its throughput only (the other ranks wait at the barrier)
        if precision == abi.POISSON_BF16X3 and args.fp32_steps > 0 and world == 1:
            v32, it32 = fp32_arm(db, args.workload, init_x, init_y, args.fp32_steps)
            line["fp32_value"] = v32
            line["fp32_iterations_per_step"] = it32
            line["bf16x3_over_fp32"] = value / world / v32
        if args.serve_leg and args.workload == "large" and world == 1:
            ep.ctx.close()
            line["serving"] = serve_leg()
        if args.cpu_baseline and world == 1:
            db.node_x[:] = init_x
            db.node_y[:] = init_y
            line["cpu_baseline"] = cpu_baseline_sample(db, args.workload)
        print(json.dumps(line))
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    return 0


# ------------------------------------------------------------------ extra studies
def blob_density(m, seed):
    """The operator sweep's density: 50 seeded Gaussian blobs (sigma U[2,40] bins, amplitude
    U[0.5,3]) on a 0.3 floor, clipped at 0 and mean-removed."""
    rng = np.random.default_rng(seed)
    c = np.arange(m, dtype=np.float64) + 0.5
    v = np.full((m, m), 0.3)
    for _ in range(50):
        cx, cy = rng.uniform(0, m, 2)
        sig = rng.uniform(2, 40)
        amp = rng.uniform(0.5, 3)
        gx = np.exp(-((c - cx) ** 2) / (2 * sig * sig))
        gy = np.exp(-((c - cy) ** 2) / (2 * sig * sig))
        v += amp * np.outer(gx, gy)
    v = np.clip(v, 0, None)
    return (v - v.mean()).astype(np.float32)


def rel_errors(ref, got):
    ref = np.asarray(ref, np.float64)
    d = np.asarray(got, np.float64) - ref
    scale = max(np.abs(ref).max(), 1e-300)
    return [float(np.abs(d).max() / scale), float(np.sqrt(np.mean(d * d)) / scale)]


def run_poisson_sweep(args):
    """Operator sweep over grid sizes and batches: device time per solve of the FP32 and the
    split-BF16 forms (L2 flushed before every timed call), algorithmic TFLOP/s (14 M^3 per
    grid) against the measured bf16 peak, and max/RMS error of phi, xi_x, xi_y against the
    FP64 form; the reference's CPU solve (FFT stand-in for FFTW) timed beside them."""
    import torch

    from superplace_b200 import engine

    _, bf16, peak_kind = peaks()
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device="cuda")  # 256 MB > L2
    s = torch.cuda.current_stream()
    for m in (128, 512, 1024, 2048):
        rho1 = blob_density(m, 1000 + m)
        ref64 = engine.PoissonBackend(m, m, 1.0, 1.0, abi.POISSON_FP64).solve(rho1)
        cpu = None
        try:
            from oracle import ref

            if ref.available():
                ref.lib().spref_set_threads(os.cpu_count() or 1)
                ref.poisson(rho1, 1.0, 1.0)
                t0 = time.perf_counter()
                for _ in range(3):
                    ref.poisson(rho1, 1.0, 1.0)
                cpu = (time.perf_counter() - t0) / 3 * 1e6
        except Exception:  # the CPU column must not hide the device numbers
            cpu = None
        for prec, name in ((abi.POISSON_FP32, "fp32"), (abi.POISSON_BF16X3, "bf16x3")):
            got = engine.PoissonBackend(m, m, 1.0, 1.0, prec).solve(rho1)
            err = {k: rel_errors(r, g) for k, r, g in zip(("phi", "xi_x", "xi_y"), ref64, got)}
            for batch in (1, 64):
                be = engine.PoissonBackend(m, m, 1.0, 1.0, prec, batch=batch)
                rho = torch.from_numpy(np.ascontiguousarray(np.broadcast_to(rho1, (batch, m, m)))).cuda()
                out = [torch.empty_like(rho) for _ in range(3)]
                call = lambda: be.solve_device(rho.data_ptr(), *(o.data_ptr() for o in out),
                                               stream=s.cuda_stream, batch=batch)
                for _ in range(3):
                    call()
                times = []
                for _ in range(10 if batch == 1 else 3):
                    flush.zero_()
                    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                    e0.record(s)
                    call()
                    e1.record(s)
                    e1.synchronize()
                    times.append(e0.elapsed_time(e1) * 1e3)
                us = statistics.median(times)
                tflops = 14.0 * m ** 3 * batch / (us * 1e-6) / 1e12
                print(json.dumps({"study": "poisson-sweep", "grid": m, "batch": batch, "precision": name,
                                  "us_per_call": us, "us_per_grid": us / batch, "grids_per_s": batch / (us * 1e-6),
                                  "tflops_algorithmic": tflops, "frac_of_bf16_peak": tflops / bf16,
                                  "peak_kind": peak_kind, "err_vs_fp64": err,
                                  "cpu_reference_us_per_grid": cpu, "cpu_cores": os.cpu_count()}), flush=True)
                del be, rho, out
                torch.cuda.empty_cache()
    return 0


def run_precision_study(args):
    """The 211k-cell mGP stage with the FP64, FP32 and split-BF16 Poisson forms and the
    reference's CPU run: iterations, final tau and HPWL, and HPWL against FP64 and CPU."""
    from superplace_b200 import engine

    db = make_design("large")
    engine.initialize_fillers(db, 1.0, 1002)
    out = {}
    for prec, name in ((abi.POISSON_FP64, "fp64"), (abi.POISSON_FP32, "fp32"), (abi.POISSON_BF16X3, "bf16x3")):
        d = db.copy()
        r = engine.EPlace(d, abi.default_params(gp_bin_dim=512, poisson_precision=prec)).run(abi.STAGE_MGP)
        out[name] = {"iterations": r.iterations, "hpwl": r.hpwl, "tau": r.overflow, "converged": r.converged,
                     "loop_ms": r.elapsed_ms}
    cpu = None
    try:
        from oracle import ref

        if ref.available():
            ref.lib().spref_set_threads(os.cpu_count() or 1)
            res, _ = ref.RefDb(db).eplace(abi.default_params(gp_bin_dim=512))
            cpu = {"iterations": int(res["iterations"]), "hpwl": res["hpwl"], "tau": res["overflow"],
                   "converged": int(res["converged"]), "loop_ms": res["elapsed_ms"]}
    except Exception as e:
        cpu = {"failed": str(e)}
    for name, v in out.items():
        v["hpwl_vs_fp64"] = v["hpwl"] / out["fp64"]["hpwl"] - 1.0
        if cpu and "hpwl" in cpu:
            v["hpwl_vs_cpu"] = v["hpwl"] / cpu["hpwl"] - 1.0
    print(json.dumps({"study": "precision", "workload": WORKLOADS["large"]["desc"], "device": out,
                      "cpu_reference": cpu, "cpu_cores": os.cpu_count()}), flush=True)
    return 0


def ref_macro_legaliser(params):
    """The reference's own legalizeMacros (oracle/_ref; src/lg/macro_sa.cpp:493) as the mLG
    callable of superplace_b200.flow.global_place: host code on the reference's side of the
    boundary, run between the device stages as GlobalPlaceStage runs it (gp_stage.cpp:128-132)."""
    from oracle import ref

    def run(db):
        r = ref.RefDb(db)
        t = time.perf_counter()
        res = r.legalize_macros(params)
        res["ms"] = (time.perf_counter() - t) * 1e3
        x, y, _, _, flags = r.nodes()
        n = db.total_nodes
        db.node_x[:n], db.node_y[:n], db.node_flags[:n] = x[:n], y[:n], flags[:n]
        return res

    return run


def run_mixed_study(args):
    """The mixed-size four-stage GP (mGP -> mLG -> FILLERONLY -> cGP) on the 211k-cell
    design with 63 movable macros (56.9% of movable area) and 200 fixed macros, 1024x1024 bins,
    with the FP64, FP32 and split-BF16 Poisson forms on the device (mLG: the reference's own SA on
    the host) and the reference's whole four-stage run on the CPU: per stage iterations, device
    loop time, HPWL and tau, and the final HPWL of each form against FP64 and the CPU run."""
    from oracle import ref
    from superplace_b200 import engine, flow

    bins = 1024
    db0 = generator.mixed_design(1002, n_cells=args.mixed_cells)
    ref.lib().spref_set_threads(os.cpu_count() or 1)
    out = {}
    for name in args.mixed_forms:
        prec = {"fp64": abi.POISSON_FP64, "fp32": abi.POISSON_FP32, "bf16x3": abi.POISSON_BF16X3}[name]
        params = abi.default_params(gp_bin_dim=bins, poisson_precision=prec)
        db = db0.copy()
        mlg = ref_macro_legaliser(params)
        after_mlg = {}

        def legalise(pdb):
            out = mlg(pdb)
            after_mlg["db"] = pdb.copy()
            return out

        t = time.perf_counter()
        res = flow.global_place(db, params, legalize_macros=legalise)
        wall = (time.perf_counter() - t) * 1e3
        o = {k: {"iterations": r.iterations, "hpwl": r.hpwl, "tau": r.overflow, "converged": r.converged,
                 "loop_ms": r.elapsed_ms} for k, r in res.items() if k in ("mGP", "FILLERONLY", "cGP")}
        o["mLG"] = res.get("mLG")
        o["stopped"] = res.get("stopped")
        o["wall_ms"] = wall
        o["final_hpwl"] = res.get("cGP", res["mGP"]).hpwl
        o["final_tau"] = res.get("cGP", res["mGP"]).overflow
        if name == args.mixed_forms[-1] and "db" in after_mlg and args.mixed_cpu:
            # FILLERONLY and cGP of the reference build from this form's own post-mLG state (the
            # same macro layout): isolates the device stages from the SA's input differences
            sdb = after_mlg["db"]
            engine.scatter_fillers(sdb, params.random_seed, seed_offset=1)
            rdb = ref.RefDb(sdb)
            same = {}
            for st, sname in ((abi.STAGE_FILLER_ONLY, "FILLERONLY"), (abi.STAGE_CGP, "cGP")):
                r_, _ = rdb.eplace(abi.default_params(gp_bin_dim=bins), stage=st)
                same[sname] = {k: r_[k] for k in ("iterations", "hpwl", "overflow", "converged", "stagnated")}
            same["cgp_hpwl_device_vs_reference"] = o["cGP"]["hpwl"] / same["cGP"]["hpwl"] - 1.0
            o["reference_from_same_mlg_state"] = same
        out[name] = o
        print(json.dumps({"study": "mixed-partial", "form": name, **o}), flush=True)
    cpu = None
    if args.mixed_cpu:
        db = db0.copy()
        ref_fillers(db, ref)
        t = time.perf_counter()
        res = ref.RefDb(db).gp_four_stage(abi.default_params(gp_bin_dim=bins))
        cpu = {**res, "wall_ms": (time.perf_counter() - t) * 1e3, "final_hpwl": res["cGP"]["hpwl"],
               "final_tau": res["cGP"]["overflow"]}
    for name, v in out.items():
        if "fp64" in out:
            v["final_hpwl_vs_fp64"] = v["final_hpwl"] / out["fp64"]["final_hpwl"] - 1.0
        if cpu:
            v["final_hpwl_vs_cpu"] = v["final_hpwl"] / cpu["final_hpwl"] - 1.0
    print(json.dumps({"study": "mixed", "workload": f"{db0.num_movable - 63} cells + 63 movable macros, "
                      f"200 fixed macros, {db0.num_nets} nets, {bins}x{bins} bins", "device": out,
                      "cpu_reference": cpu, "cpu_cores": os.cpu_count()}), flush=True)
    return 0


def serve_leg(rate=200.0, seconds=1.5, n_designs=16, slots=8):
    """A short leg of the serving study for the bench line (the study's highest rate, 200 req/s):
    requests from the serving generator (cells log-uniform in 1k..100k) arriving as a Poisson
    process at `rate` per second for about `seconds`, served by `slots` slots, against the same
    trace placed one at a time with plain-FP32 solves. placements/s, p50/p99 latency from
    arrival to the converged placement, and p99 against the median single plain-FP32 solve on
    an idle device and against the p99 of the same requests placed alone."""
    from superplace_b200 import engine, generator, serving

    rng = np.random.default_rng(11)
    designs = []
    for i in range(n_designs):
        n = int(round(np.exp(rng.uniform(np.log(1e3), np.log(1e5)))))
        db, grid = generator.scaled_design(5000 + i, n)
        engine.initialize_fillers(db, 1.0, 1002)
        designs.append((db, grid))
    by_grid = {}
    for d in designs:
        by_grid.setdefault(d[1], d)

    def warm(srv, k):
        for req in by_grid.values():
            for f in [srv.submit(*req) for _ in range(k)]:
                f.result()

    with serving.PlacementServer(slots=1, precision="fp32") as srv:
        warm(srv, 1)
        single = [srv.submit(db, g).result().latency for db, g in designs]
    with serving.PlacementServer(slots=1) as srv:  # the server's own form, alone on the device
        warm(srv, 1)
        alone = [srv.submit(db, g).result().latency for db, g in designs]
    n = max(16, int(rate * seconds))
    arrivals = serving.poisson_arrivals(rate, n, seed=int(rate))
    reqs = [designs[i % n_designs] for i in range(n)]
    with serving.PlacementServer(slots=slots, hbm_budget_bytes=150e9) as srv:
        warm(srv, slots)
        ours = serving.summarize(serving.replay(srv, reqs, arrivals))
    with serving.PlacementServer(slots=1, precision="fp32") as srv:
        warm(srv, 1)
        base = serving.summarize(serving.replay(srv, reqs, arrivals))
    single_ms = float(np.median(single) * 1e3)
    solo_p99_ms = float(np.percentile([alone[i % n_designs] for i in range(n)], 99) * 1e3)
    return {"rate_per_s": rate, "requests": n, "slots": slots, "designs": n_designs,
            "placements_per_s": ours["placements_per_s"], "p50_ms": ours["p50_ms"], "p99_ms": ours["p99_ms"],
            "one_at_a_time_fp32_placements_per_s": base["placements_per_s"],
            "one_at_a_time_fp32_p99_ms": base["p99_ms"],
            "throughput_ratio": ours["placements_per_s"] / base["placements_per_s"],
            "single_fp32_solve_median_ms": single_ms, "p99_over_single_solve": ours["p99_ms"] / single_ms,
            "solo_p99_ms": solo_p99_ms, "p99_over_solo_p99": ours["p99_ms"] / solo_p99_ms,
            "converged": ours["converged"]}


def run_serve(args):
    """The serving loop on arrival traces: requests from the small generator (cells log-uniform
    in 1k..100k, nets 1.05x cells, grid the next power of two in 64..512 at ~4 cells per bin),
    Poisson arrivals at 10, 50 and 200 req/s, admitted against a 150 GB budget. The server
    (`--slots` slots, split-BF16 where the grid tiles by 128) is compared with one-at-a-time
    plain-FP32 solves on the same trace: placements/s and p50/p99 latency from arrival to the
    converged placement. Distinct designs are generated once and reused across the trace."""
    from superplace_b200 import engine, generator, serving

    rng = np.random.default_rng(11)
    n_distinct = args.serve_designs
    designs = []
    for i in range(n_distinct):
        n = int(round(np.exp(rng.uniform(np.log(1e3), np.log(1e5)))))
        db, grid = generator.scaled_design(5000 + i, n)
        engine.initialize_fillers(db, 1.0, 1002)
        designs.append((db, grid))
    # each design's solve time alone on an idle device (the server's own form, warmed slot):
    # the reference of every request's slowdown in the mix
    alone = {}
    with serving.PlacementServer(slots=1) as srv:
        for f in [srv.submit(db, g) for db, g in designs[:4]]:
            f.result()
        for i, (db, g) in enumerate(designs):
            alone[i] = srv.submit(db, g).result().latency
    single_fp32 = []
    with serving.PlacementServer(slots=1, precision="fp32") as srv:
        for db, g in designs[:16]:
            single_fp32.append(srv.submit(db, g).result().latency)
    single = {"fp32_median_ms": float(np.median(single_fp32) * 1e3),
              "server_form_median_ms": float(np.median(list(alone.values())) * 1e3)}

    by_grid = {}
    for db, g in designs:
        by_grid.setdefault(g, (db, g))

    def warm(srv, k):
        # a long-running server: every slot has placed a request of each grid size before the
        # trace starts (so each holds its Poisson plans and loop graph)
        for req in by_grid.values():
            for f in [srv.submit(*req) for _ in range(k)]:
                f.result()

    for rate in args.serve_rates:
        n = min(512, max(16, int(rate * args.serve_seconds)))
        arrivals = serving.poisson_arrivals(rate, n, seed=int(rate))
        idx = [i % n_distinct for i in range(n)]
        reqs = [designs[i] for i in idx]
        with serving.PlacementServer(slots=args.slots, hbm_budget_bytes=150e9) as srv:
            warm(srv, args.slots)
            res = serving.replay(srv, reqs, arrivals)
            ours = serving.summarize(res)
            ours["peak_running"] = srv.peak_running
            slow = np.array([r.latency / alone[i] for r, i in zip(res, idx)])
            solo = np.array([alone[i] for i in idx])
            ours["slowdown_vs_alone"] = {"p50": float(np.percentile(slow, 50)), "p99": float(np.percentile(slow, 99))}
            # the trace's p99 latency against the p99 of the same requests' solo latencies
            ours["p99_over_solo_p99"] = float(np.percentile([r.latency for r in res], 99) /
                                             np.percentile(solo, 99))
        with serving.PlacementServer(slots=1, precision="fp32") as srv:
            warm(srv, 1)
            base = serving.summarize(serving.replay(srv, reqs, arrivals))
        print(json.dumps({"study": "serve", "rate_per_s": rate, "requests": n, "slots": args.slots,
                          "ours": ours, "one_at_a_time_fp32": base,
                          "throughput_ratio": ours["placements_per_s"] / base["placements_per_s"],
                          "single_solve_ms": single,
                          "p99_over_single_fp32": ours["p99_ms"] / single["fp32_median_ms"],
                          "designs": n_distinct, "data": "synthetic"}), flush=True)
    return 0


def run_bookshelf(args):
    """BookShelf I/O on the 211k-cell design written as BookShelf files: the engine library's
    reader and .pl writer against the reference's own BookshelfReader / BookshelfWriter
    (oracle/_ref, single-threaded as shipped). Host work only; one JSON line."""
    import tempfile

    from superplace_b200 import bookshelf
    db = make_design("large")
    d = tempfile.mkdtemp(prefix="spg_bookshelf_")
    aux = bookshelf.write_bookshelf(d, "large", db)
    size = sum(os.path.getsize(os.path.join(d, f)) for f in os.listdir(d))
    reps = max(3, args.steps)

    def med(fn):
        fn()  # warm the page cache
        ts = []
        for _ in range(reps):
            t = time.perf_counter()
            fn()
            ts.append((time.perf_counter() - t) * 1e3)
        return statistics.median(ts)

    rd = bookshelf.read_bookshelf(aux)
    line = {"study": "bookshelf", "design": "211k cells, 221k nets, 859k pins (synthetic)",
            "bytes": size, "threads": len(os.sched_getaffinity(0)), "reps": reps,
            "read_ms": round(med(lambda: bookshelf.read_bookshelf(aux)), 2),
            "write_pl_ms": round(med(lambda: bookshelf.write_pl(os.path.join(d, "o.pl"), rd)), 2)}
    from oracle import ref
    if ref.available():
        r = ref.bookshelf_read(aux)
        line["ref_read_ms"] = round(med(lambda: ref.bookshelf_read(aux)), 2)
        line["ref_write_pl_ms"] = round(med(lambda: ref.write_pl(r, os.path.join(d, "r.pl"))), 2)
        line["read_speedup"] = round(line["ref_read_ms"] / line["read_ms"], 2)
        line["write_pl_speedup"] = round(line["ref_write_pl_ms"] / line["write_pl_ms"], 2)
    for f in os.listdir(d):
        os.remove(os.path.join(d, f))
    os.rmdir(d)
    print(json.dumps(line))
    return 0


def run_qp(args):
    """B2B quadratic initial placement of the 211k-cell design (QuadraticPlacer::place with
    configs/default.json's QP keys): the system assembled on the host, BiCGSTAB on the host
    (all threads) and on the GPU. Both give the same bits; one JSON line. The reference's own
    QP needs Eigen, which is not installed here, so it has no arm."""
    from superplace_b200 import qp
    db = make_design("large")
    line = {"study": "qp", "design": "211k cells, 221k nets, 859k pins (synthetic)",
            "threads": len(os.sched_getaffinity(0))}
    # CUDA start-up (context, modules) outside the timed runs: one small device placement first
    small = make_design("small")
    qp.QuadraticPlacer(qp.default_params(device=1, max_iter=1)).place(small)
    res = {}
    for name, dev in (("host", 0), ("device", 1)):
        a = db.copy()
        t = time.perf_counter()
        rows = qp.QuadraticPlacer(qp.default_params(device=dev)).place(a)
        res[name] = (a, rows, (time.perf_counter() - t) * 1e3)
        line[f"{name}_ms"] = round(res[name][2], 1)
        line[f"{name}_ms_per_outer_iter"] = [round(v, 1) for v in rows["elapsed_ms"]]
        line[f"{name}_assemble_ms"] = round(float(np.sum(rows["assemble_ms"])), 1)
        line[f"{name}_solve_ms"] = round(float(np.sum(rows["solve_ms"])), 1)
    (ha, hr, _), (da, dr, _) = res["host"], res["device"]
    line["outer_iters"] = int(dr["iter"].shape[0])
    line["solver_iters"] = [int(v) for v in dr["solver_iters_x"]] + [int(v) for v in dr["solver_iters_y"]]
    line["final_hpwl"] = float(dr["hpwl"][-1])
    line["device_equals_host"] = bool(np.array_equal(da.node_x, ha.node_x) and np.array_equal(da.node_y, ha.node_y))
    line["speedup"] = round(line["host_ms"] / line["device_ms"], 2)
    print(json.dumps(line))
    return 0


def run_flow(args):
    """The whole pipeline on the 211k design written as BookShelf files: parse, QP init, mGP
    (fillers and the device loop) and the .pl write through superplace_b200.flow, with the lg
    stage the reference's own legalizeCells on its side of the boundary (oracle/_ref, passed to
    the flow as its cell legaliser); and the reference's own stages on the same files
    (oracle/_ref: its reader, initializeFillers, EPlace mGP, legalizeCells, writePl; its QP needs
    Eigen, so it starts from our QP result). Wall times per stage and HPWL after each; one JSON
    line."""
    import tempfile

    from oracle import ref
    from superplace_b200 import bookshelf, flow
    db0 = make_design("large")
    d = tempfile.mkdtemp(prefix="spg_flow_")
    aux = bookshelf.write_bookshelf(d, "large", db0)
    # CUDA start-up outside the timed runs
    flow.place(db=make_design("small"), stages=("init", "gp"))
    params = abi.default_params(gp_bin_dim=WORKLOADS["large"]["bin_dim"], poisson_precision=abi.POISSON_BF16X3)
    def legalize_cells(pdb):
        r = ref.RefDb(pdb)
        res = ref.abacus(r)
        x, y, _, _, _ = r.nodes()
        pdb.node_x[: pdb.total_nodes], pdb.node_y[: pdb.total_nodes] = x, y
        return res

    db, rep = flow.place(aux, out_pl=os.path.join(d, "ours.pl"), params=params, legalize_cells=legalize_cells)
    ours = {s["stage"]: {k: (round(v, 3) if isinstance(v, float) else v) for k, v in s.items() if k != "stage"}
            for s in rep["stages"]}
    line = {"study": "flow", "design": "211k cells, 221k nets, 859k pins (synthetic), 512x512 bins",
            "threads": len(os.sched_getaffinity(0)), "ours": ours,
            "ours_total_ms": round(sum(s["ms"] for s in rep["stages"]), 1)}
    if ref.available():
        theirs = {}
        t = time.perf_counter()
        r = ref.bookshelf_read(aux)
        theirs["parse"] = {"ms": round((time.perf_counter() - t) * 1e3, 1)}
        x = np.zeros(r.counts()[1], np.float32)
        y = np.zeros_like(x)
        x[:], y[:] = rep["init_x"], rep["init_y"]
        r.set_xy(x, y)
        t = time.perf_counter()
        r.fillers_init(1.0, 1002)
        ref.lib().spref_set_threads(len(os.sched_getaffinity(0)))
        res, _ = r.eplace(abi.default_params(gp_bin_dim=WORKLOADS["large"]["bin_dim"]), abi.STAGE_MGP)
        theirs["gp"] = {"ms": round((time.perf_counter() - t) * 1e3, 1), "iterations": int(res["iterations"]),
                        "hpwl": res["hpwl"], "overflow": res["overflow"]}
        t = time.perf_counter()
        lg = ref.abacus(r)
        theirs["lg"] = {"ms": round((time.perf_counter() - t) * 1e3, 1), "hpwl": r.hpwl(), "failed": lg["failed"],
                        "disp_mean": lg["disp_mean"]}
        t = time.perf_counter()
        ref.write_pl(r, os.path.join(d, "ref.pl"))
        theirs["write"] = {"ms": round((time.perf_counter() - t) * 1e3, 1)}
        if os.path.exists(ref.CHECK_PATH):  # the reference's legality checker on both outputs
            line["ours_check"] = "PASS" if ref.check_placement(aux, os.path.join(d, "ours.pl"))[0] == 0 else "FAIL"
            theirs["check"] = "PASS" if ref.check_placement(aux, os.path.join(d, "ref.pl"))[0] == 0 else "FAIL"
        line["reference"] = theirs
        line["reference_note"] = "init: the reference's QP needs Eigen (absent); it starts from our QP placement"
        line["reference_total_ms_without_init"] = round(sum(v["ms"] for v in theirs.values() if isinstance(v, dict)), 1)
        line["ours_total_ms_without_init"] = round(line["ours_total_ms"] - ours["init"]["ms"], 1)
    for f in os.listdir(d):
        os.remove(os.path.join(d, f))
    os.rmdir(d)
    print(json.dumps(line))
    return 0


def run_stage_once(args):
    """One mGP stage of the workload (its instance, fillers and grid) through the public API,
    for profilers: the loop's kernels in their order, nothing else timed or printed but one
    line. Under ncu, set SPG_HOST_LOOP=1 (ncu does not profile kernels inside conditional graphs)
    and SPG_TC_TUNE=0 (the tile-shape tuner's timing is distorted under the profiler)."""
    from superplace_b200 import engine

    db = make_design(args.workload)
    engine.initialize_fillers(db, 1.0, 1002)
    precision = abi.POISSON_BF16X3 if args.precision == "bf16x3" else abi.POISSON_FP32
    params = abi.default_params(gp_bin_dim=WORKLOADS[args.workload]["bin_dim"], poisson_precision=precision)
    r = engine.EPlace(db, params).run(abi.STAGE_MGP)
    print(json.dumps({"stage": "mGP", "iterations": r.iterations, "hpwl": r.hpwl, "overflow": r.overflow}))
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--precision", default="bf16x3", choices=["fp32", "bf16x3"])
    ap.add_argument("--workload", default="large", choices=list(WORKLOADS))
    ap.add_argument("--ref-iters", type=int, default=0,
                    help="reference arm: time only the first N mGP iterations of each stage (0: full stages)")
    ap.add_argument("--no-cpu-baseline", dest="cpu_baseline", action="store_false")
    ap.add_argument("--no-serve-leg", dest="serve_leg", action="store_false",
                    help="leave out the short serving leg (200 req/s) of the bench line")
    ap.add_argument("--fp32-steps", type=int, default=3,
                    help="stages of the plain FP32 form timed after the headline arm (fp32_value)")
    ap.add_argument("--poisson-sweep", action="store_true",
                    help="operator sweep (grids 128..2048, batch 1 and 64): JSON lines, not the bench line")
    ap.add_argument("--precision-study", action="store_true",
                    help="211k mGP with FP64 / FP32 / BF16x3 Poisson and the CPU reference: one JSON line")
    ap.add_argument("--serve", action="store_true",
                    help="serving loop on Poisson arrival traces: JSON lines, not the bench line")
    ap.add_argument("--bookshelf", action="store_true",
                    help="BookShelf read / .pl write on the 211k design against the reference's: one JSON line")
    ap.add_argument("--qp", action="store_true",
                    help="B2B quadratic initial placement of the 211k design, host vs GPU solver: one JSON line")
    ap.add_argument("--flow", action="store_true",
                    help="parse, QP init, mGP, Abacus and .pl write on the 211k design, ours and the reference's: one JSON line")
    ap.add_argument("--mixed-study", action="store_true",
                    help="four-stage mixed-size GP (211k cells + 63 movable macros) at 1024x1024 bins, "
                         "FP64/FP32/BF16x3 and the CPU run: JSON lines")
    ap.add_argument("--mixed-cells", type=int, default=211_000)
    ap.add_argument("--mixed-forms", nargs="+", default=["fp64", "fp32", "bf16x3"])
    ap.add_argument("--no-mixed-cpu", dest="mixed_cpu", action="store_false")
    ap.add_argument("--stage-once", action="store_true",
                    help="one mGP stage of the workload at --precision, no timing (the profiles' command)")
    ap.add_argument("--slots", type=int, default=8)
    ap.add_argument("--serve-rates", type=float, nargs="+", default=[10.0, 50.0, 200.0])
    ap.add_argument("--serve-seconds", type=float, default=8.0)
    ap.add_argument("--serve-designs", type=int, default=48)
    args = ap.parse_args()
    # the serving study and the bench line's serving leg run 8 slots of two streams each: give
    # the device as many hardware work queues (read when the CUDA context is created, which has
    # not happened yet in this process)
    os.environ.setdefault("CUDA_DEVICE_MAX_CONNECTIONS", "16")
    if args.stage_once:
        return run_stage_once(args)
    if args.serve:
        return run_serve(args)
    if args.poisson_sweep:
        return run_poisson_sweep(args)
    if args.bookshelf:
        return run_bookshelf(args)
    if args.qp:
        return run_qp(args)
    if args.flow:
        return run_flow(args)
    if args.precision_study:
        return run_precision_study(args)
    if args.mixed_study:
        return run_mixed_study(args)
    if args.impl == "reference":
        return run_reference(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
