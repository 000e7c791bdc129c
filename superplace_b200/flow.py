"""The GP stage and the reference's placement pipeline (src/main.cpp:55-115) over this package.

  parse  read_bookshelf                 BookshelfReader::read
  init   QuadraticPlacer (B2B QP)       makeInitialPlacer("quadratic"), the default init_method
  gp     global_place                   GlobalPlaceStage::run (src/stages/gp_stage.cpp:59-244)
  lg     the caller's cell legaliser    LegalizeStage::run (src/stages/lg_stage.cpp:12-41)
  write  write_pl                       BookshelfWriter::writePl

Macro legalisation (mLG, the reference's simulated annealing, src/lg/macro_sa.cpp:493) and
cell legalisation (Abacus, src/lg/abacus.cpp:155) stay host code on the reference's side of
the boundary: the caller passes them in as callables over the PlaceDB, the way
GlobalPlaceStage and the pipeline call them between the device stages. Without an mLG
callable a design with movable macros stops after mGP; without a cell legaliser the lg stage
is skipped.
"""
from __future__ import annotations

import time
from dataclasses import dataclass
from typing import Callable

import numpy as np

from . import abi, bookshelf, engine, qp
from .placedb import F_FIXED, F_MACRO, PlaceDB

STAGES = ("parse", "init", "gp", "lg", "write")

Legaliser = Callable[[PlaceDB], dict]


@dataclass
class FrameMark:
    """FrameMark (src/util/metrics.h:31-37): a moment of the run worth a frame. `t` is the GP
    iteration count accumulated over mGP, FILLERONLY and cGP (the playback clock), `iter` -1 marks
    a stage milestone, `break_before` a jump the player must not interpolate across."""
    stage: str
    iter: int
    t: float
    break_before: bool
    label: str


# the frame hook: (mark, x, y) with every node's position at that moment (MetricsSink's
# FrameHook, src/util/metrics.h:67-71; the PlaceDB itself is not updated inside a stage)
FrameHook = Callable[[FrameMark, np.ndarray, np.ndarray], None]


def _hpwl(db: PlaceDB) -> float:
    return qp.host_hpwl(db)


def movable_macros(db: PlaceDB) -> np.ndarray:
    """Indices of the movable macros not yet fixed (GlobalPlaceStage's count, gp_stage.cpp:80-84)."""
    f = db.node_flags[: db.num_movable]
    return np.nonzero(((f & F_MACRO) != 0) & ((f & F_FIXED) == 0))[0]


def global_place(db: PlaceDB, params: abi.Params | None = None, legalize_macros: Legaliser | None = None,
                 metrics: list | None = None, frame_hook: FrameHook | None = None, frame_stride: int = 0,
                 diagnostics: str | None = None) -> dict:
    """GlobalPlaceStage::run (src/stages/gp_stage.cpp:59-244) on the device: fillers, mGP, then
    for designs with movable macros mLG (the caller's `legalize_macros`, which must leave every
    macro F_FIXED), fillers re-scattered with seed offset 1, FILLERONLY and cGP. The positions
    of the frozen macros are checked bit for bit after cGP (gp_stage.cpp:205-225). Returns each
    stage's result (abi.Result) and, with mLG, the legaliser's report; `stopped` says why the
    sequence ended early.

    frame_hook with frame_stride > 0 gets the reference's frame marks (gp_stage.cpp:73-93,136):
    every frame_stride-th iteration of each stage, the end of mGP and of cGP (a break when the
    stage rolled back), and mLG. `diagnostics`: the output directory of the GP diagnostics of
    mGP and cGP (Config::gp_diagnostics)."""
    p = params or abi.default_params()
    out: dict = {}
    t_offset = [0.0]
    hook = frame_hook if frame_hook is not None and frame_stride > 0 else None
    engine.initialize_fillers(db, p.target_density, p.random_seed)
    ep = engine.EPlace(db, p)
    if hook:
        names = {abi.STAGE_MGP: "mGP", abi.STAGE_FILLER_ONLY: "FILLERONLY", abi.STAGE_CGP: "cGP"}
        ep.set_iter_callback(lambda st, it, x, y: hook(
            FrameMark(names[st], it, t_offset[0] + it, False, f"{names[st]} iter {it}"), x, y), frame_stride)

    def mark_end(name, r):
        if hook:
            label = (f"{name} end (tau stagnated, rolled back to iteration {r.rollback_iter})" if r.stagnated
                     else f"{name} end")
            hook(FrameMark(name, r.iterations, t_offset[0], bool(r.stagnated), label), db.node_x, db.node_y)

    out["mGP"] = ep.run(abi.STAGE_MGP, metrics, diagnostics)
    t_offset[0] = float(out["mGP"].iterations)
    mark_end("mGP", out["mGP"])
    macros = movable_macros(db)
    if macros.size == 0:
        return out
    if legalize_macros is None:
        out["stopped"] = f"{macros.size} movable macros need mLG and no macro legaliser was given; stopped after mGP"
        return out
    out["mLG"] = legalize_macros(db)
    if np.any((db.node_flags[macros] & F_FIXED) == 0):
        raise engine.SpgError(abi.SPG_E_STATE, "mLG left a movable macro unfixed")
    if hook:
        hook(FrameMark("mLG", -1, t_offset[0], True, "mLG macro legalisation (macros moved to legal sites)"),
             db.node_x, db.node_y)
    mx, my = db.node_x[macros].copy(), db.node_y[macros].copy()
    engine.scatter_fillers(db, p.random_seed, seed_offset=1)
    out["FILLERONLY"] = ep.run(abi.STAGE_FILLER_ONLY, metrics, diagnostics)
    t_offset[0] += out["FILLERONLY"].iterations
    out["cGP"] = ep.run(abi.STAGE_CGP, metrics, diagnostics)
    t_offset[0] += out["cGP"].iterations
    mark_end("cGP", out["cGP"])
    if not (np.array_equal(db.node_x[macros], mx) and np.array_equal(db.node_y[macros], my)):
        raise engine.SpgError(abi.SPG_E_STATE, "a frozen macro changed position during cGP")
    return out


def place(aux: str | None = None, db: PlaceDB | None = None, out_pl: str | None = None,
          stages=STAGES, params: abi.Params | None = None, qp_params=None,
          legalize_macros: Legaliser | None = None, legalize_cells: Legaliser | None = None) -> tuple[PlaceDB, dict]:
    """Runs `stages` in order on the design of `aux` (or on `db`) and returns the PlaceDB and a
    report: per stage its wall time in ms and the HPWL after it, the GP and legalisation
    results, and `stopped` when a stage could not run."""
    report = {"stages": []}

    def done(name, t0, **extra):
        report["stages"].append(dict(stage=name, ms=(time.perf_counter() - t0) * 1e3, hpwl=_hpwl(db), **extra))

    if "parse" in stages:
        t0 = time.perf_counter()
        db = bookshelf.read_bookshelf(aux)
        done("parse", t0, nodes=db.num_nodes, movable=db.num_movable, nets=db.num_nets, pins=db.num_pins)
    if db is None:
        raise ValueError("no design: give aux with the parse stage, or db")
    if "init" in stages:
        t0 = time.perf_counter()
        qp_params = qp_params or qp.default_params(device=1 if engine.device_available() else 0)
        rows = qp.QuadraticPlacer(qp_params).place(db)
        done("init", t0, outer_iters=int(rows["iter"].shape[0]), device=int(qp_params.device))
        report["init_x"], report["init_y"] = db.node_x[: db.num_nodes].copy(), db.node_y[: db.num_nodes].copy()
    if "gp" in stages:
        t0 = time.perf_counter()
        res = global_place(db, params, legalize_macros)
        last = res.get("cGP", res["mGP"])
        done("gp", t0, iterations=sum(r.iterations for k, r in res.items() if k in ("mGP", "FILLERONLY", "cGP")),
             overflow=last.overflow, loop_ms=sum(r.elapsed_ms for k, r in res.items() if k in ("mGP", "FILLERONLY", "cGP")))
        if "stopped" in res:
            report["stopped"] = res["stopped"]
            return db, report
    if "lg" in stages and legalize_cells is not None:
        t0 = time.perf_counter()
        done("lg", t0, **legalize_cells(db))
    if "write" in stages and out_pl:
        t0 = time.perf_counter()
        bookshelf.write_pl(out_pl, db)
        done("write", t0)
    return db, report
