"""The reference's placement pipeline (src/main.cpp:55-115; stages parse, init, gp, lg and the
.pl write) over this package:

  parse  read_bookshelf                 BookshelfReader::read
  init   QuadraticPlacer (B2B QP)       makeInitialPlacer("quadratic"), the default init_method;
                                        "random", "cluster_fc", "cluster_bc" by init_method
  gp     fillers + the device mGP loop  GlobalPlaceStage::run (src/stages/gp_stage.cpp)
  lg     Abacus                         LegalizeStage::run (src/stages/lg_stage.cpp:12-41)
  write  write_pl                       BookshelfWriter::writePl

GlobalPlaceStage runs only mGP when no movable macro exists (src/stages/gp_stage.cpp:114-117).
With movable macros it needs macro legalisation (mLG), which this package does not provide:
the flow stops after mGP and says so in the report.
"""
from __future__ import annotations

import time

import numpy as np

from . import abi, bookshelf, engine, initial, legalize, qp, stats
from .placedb import F_FIXED, F_MACRO, PlaceDB

STAGES = ("parse", "init", "gp", "lg", "write")


def _hpwl(db: PlaceDB) -> float:
    return qp.host_hpwl(db)


def place(aux: str | None = None, db: PlaceDB | None = None, out_pl: str | None = None,
          stages=STAGES, params: abi.Params | None = None, qp_params=None,
          init_method: str = "quadratic") -> tuple[PlaceDB, dict]:
    """Runs `stages` in order on the design of `aux` (or on `db`) and returns the PlaceDB and a
    report: per stage its wall time in ms and the HPWL after it, the GP and legalisation
    results, and `stopped` when a stage could not run."""
    report = {"stages": []}

    def done(name, t0, **extra):
        report["stages"].append(dict(stage=name, ms=(time.perf_counter() - t0) * 1e3, hpwl=_hpwl(db), **extra))

    if "parse" in stages:
        t0 = time.perf_counter()
        db = bookshelf.read_bookshelf(aux)
        st = stats.db_stats(db)
        done("parse", t0, nodes=st.node_count, fixed=st.fixed_count, macros=st.macro_count, nets=st.net_count,
             pins=st.pin_count)
        report["summary"] = stats.summary_text(st)
    if db is None:
        raise ValueError("no design: give aux with the parse stage, or db")
    if "init" in stages:
        t0 = time.perf_counter()
        if init_method == "quadratic":
            qp_params = qp_params or qp.default_params(device=1 if engine.device_available() else 0)
            rows = qp.QuadraticPlacer(qp_params).place(db)
            done("init", t0, outer_iters=int(rows["iter"].shape[0]), device=int(qp_params.device))
        else:
            seed = (params or abi.default_params()).random_seed
            done("init", t0, **initial.make_initial_placer(init_method, seed=seed).place(db))
        report["init_x"], report["init_y"] = db.node_x[: db.num_nodes].copy(), db.node_y[: db.num_nodes].copy()
    movable_macros = int(np.sum((db.node_flags[: db.num_movable] & F_MACRO != 0) &
                                (db.node_flags[: db.num_movable] & F_FIXED == 0)))
    if "gp" in stages:
        t0 = time.perf_counter()
        p = params or abi.default_params()
        engine.initialize_fillers(db, p.target_density, p.random_seed)
        ep = engine.EPlace(db, p)
        r = ep.run(abi.STAGE_MGP)
        del ep
        done("gp", t0, iterations=r.iterations, overflow=r.overflow, loop_ms=r.elapsed_ms)
        if movable_macros:
            report["stopped"] = f"{movable_macros} movable macros need mLG, which is not built; stopped after mGP"
            return db, report
    if "lg" in stages:
        t0 = time.perf_counter()
        res = legalize.legalize_cells(db)
        done("lg", t0, **res)
    if "write" in stages and out_pl:
        t0 = time.perf_counter()
        bookshelf.write_pl(out_pl, db)
        done("write", t0)
    return db, report
