"""Abacus row legalisation of the standard cells (LegalizeStage, src/stages/lg_stage.cpp:12-41,
over legalizeCells, src/lg/abacus.cpp:155-284) through the engine library's host entry point
spg_abacus_legalize.

`legalize_cells(db)` moves the PlaceDB's cells onto the rows in place and returns the
reference's AbacusResult fields; `abacus_segments(db)` lists the free row segments.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import abi
from .engine import SpgError, lib
from .placedb import PlaceDB

FIELDS = ("precondition_ok", "cells", "failed", "rows", "segments", "rounded_widths", "selfcheck_overlaps",
          "selfcheck_off_site", "disp_mean", "disp_max")


class AbacusResult(C.Structure):
    _fields_ = [(f, C.c_int32) for f in FIELDS[:8]] + [("disp_mean", C.c_double), ("disp_max", C.c_double)]


def _bind():
    L = lib()
    if not getattr(L, "_lg_bound", False):
        fp, ip = C.POINTER(C.c_float), C.POINTER(C.c_int32)
        L.spg_abacus_last_error.restype = C.c_char_p
        L.spg_abacus_legalize.argtypes = [C.POINTER(abi.DbView), C.c_int32, fp, fp, C.POINTER(AbacusResult)]
        L.spg_abacus_segments.argtypes = [C.POINTER(abi.DbView), fp, fp, ip, fp, fp, C.c_int32, ip]
        L._lg_bound = True
    return L


def _check(rc):
    if rc != 0:
        raise SpgError(rc, _bind().spg_abacus_last_error().decode())


def legalize_cells(db: PlaceDB, area_weight: bool = False) -> dict:
    view = db.view()
    res = AbacusResult()
    _check(_bind().spg_abacus_legalize(C.byref(view), int(area_weight), abi.fptr(db.node_x), abi.fptr(db.node_y),
                                       C.byref(res)))
    return {f: getattr(res, f) for f in FIELDS}


def abacus_segments(db: PlaceDB):
    view = db.view()
    n = C.c_int32(0)
    L = _bind()
    _check(L.spg_abacus_segments(C.byref(view), abi.fptr(db.node_x), abi.fptr(db.node_y), None, None, None, 0,
                                 C.byref(n)))
    row, lx, hx = np.zeros(n.value, np.int32), np.zeros(n.value, np.float32), np.zeros(n.value, np.float32)
    _check(L.spg_abacus_segments(C.byref(view), abi.fptr(db.node_x), abi.fptr(db.node_y), abi.iptr(row),
                                 abi.fptr(lx), abi.fptr(hx), n.value, C.byref(n)))
    return row, lx, hx
