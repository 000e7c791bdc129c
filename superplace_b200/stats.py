"""The parse stage's design summary, DbStats (src/db/db_stats.h:17-86), over the engine library's
host entry points spg_db_stats_compute / spg_db_stats_text."""
from __future__ import annotations

import ctypes as C

from . import abi
from .engine import lib
from .placedb import PlaceDB


class DbStats(C.Structure):
    _fields_ = [("core_lx", C.c_double), ("core_ly", C.c_double), ("core_hx", C.c_double), ("core_hy", C.c_double),
                ("row_height", C.c_double), ("row_count", C.c_int32), ("site_step", C.c_double),
                ("core_area", C.c_double), ("movable_area", C.c_double), ("fixed_area", C.c_double),
                ("fixed_area_in_core", C.c_double), ("total_row_area", C.c_double), ("node_count", C.c_int32),
                ("object_count", C.c_int32), ("fixed_count", C.c_int32), ("macro_count", C.c_int32),
                ("net_count", C.c_int32), ("pin_count", C.c_int32), ("max_net_degree", C.c_int32),
                ("degree_histogram", C.c_int32 * 5), ("degree_count", C.c_int32 * 101), ("degree_over", C.c_int32)]


def _bind():
    L = lib()
    if not getattr(L, "_stats_bound", False):
        L.spg_db_stats_compute.argtypes = [C.POINTER(abi.DbView), C.POINTER(DbStats)]
        L.spg_db_stats_text.argtypes = [C.POINTER(DbStats), C.c_char_p, C.c_int64]
        L.spg_db_stats_text.restype = C.c_int64
        L._stats_bound = True
    return L


def db_stats(db: PlaceDB) -> DbStats:
    view = db.view()
    s = DbStats()
    if _bind().spg_db_stats_compute(C.byref(view), C.byref(s)) != 0:
        raise ValueError("spg_db_stats_compute: bad PlaceDB view")
    return s


def summary_text(s: DbStats) -> str:
    """The reference's "DATABASE SUMMARY" block for these statistics."""
    L = _bind()
    n = L.spg_db_stats_text(C.byref(s), None, 0)
    buf = C.create_string_buffer(int(n) + 1)
    L.spg_db_stats_text(C.byref(s), buf, n + 1)
    return buf.value.decode()
