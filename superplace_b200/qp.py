"""B2B (Kraftwerk2) quadratic initial placement: QuadraticPlacer::place
(src/init/quadratic_placer.cpp:153-228) over the engine library's host entry point spg_qp_place.

`QuadraticPlacer().place(db)` moves the PlaceDB's movable nodes in place and returns one row per
outer iteration (iter, hpwl, err = the larger solver error, elapsed_ms, solver iterations per
axis), the reference's IterMetrics rows of the QP stage.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import abi
from .engine import SpgError, lib
from .placedb import PlaceDB


class QpParams(C.Structure):
    _fields_ = [("max_iter", C.c_int32), ("tol", C.c_float), ("solver_max_iter", C.c_int32),
                ("outer_tol", C.c_float), ("min_distance", C.c_float), ("ignore_net_degree", C.c_int32),
                ("threads", C.c_int32), ("device", C.c_int32)]


class QpRow(C.Structure):
    _fields_ = [("iter", C.c_int32), ("solver_iters_x", C.c_int32), ("solver_iters_y", C.c_int32),
                ("err", C.c_float), ("hpwl", C.c_double), ("elapsed_ms", C.c_double),
                ("assemble_ms", C.c_double), ("solve_ms", C.c_double)]


def _bind():
    L = lib()
    if not getattr(L, "_qp_bound", False):
        vp, fp, ip = C.c_void_p, C.POINTER(C.c_float), C.POINTER(C.c_int32)
        L.spg_qp_default_params.argtypes = [C.POINTER(QpParams)]
        L.spg_qp_last_error.restype = C.c_char_p
        L.spg_qp_place.argtypes = [C.POINTER(abi.DbView), vp, C.POINTER(QpParams), fp, fp, C.POINTER(QpRow),
                                   C.c_int32, ip]
        L.spg_qp_assemble.argtypes = [C.POINTER(abi.DbView), vp, C.POINTER(QpParams), C.c_int32, fp, fp, ip, ip,
                                      fp, fp, C.c_int64, C.POINTER(C.c_int64)]
        L.spg_host_hpwl.argtypes = [C.POINTER(abi.DbView), fp, fp, C.POINTER(C.c_double)]
        L._qp_bound = True
    return L


def _check(rc):
    if rc != 0:
        raise SpgError(rc, _bind().spg_qp_last_error().decode())


def default_params(**overrides) -> QpParams:
    """configs/default.json's QP keys (qp_max_iter 20, qp_tol 1e-6, qp_solver_max_iter 100,
    qp_outer_tol 1e-4, qp_min_distance 1.0, ignore_net_degree 100)."""
    p = QpParams()
    _bind().spg_qp_default_params(C.byref(p))
    for k, v in overrides.items():
        if not hasattr(p, k):
            raise KeyError(k)
        setattr(p, k, v)
    return p


def _weights(db, net_weight):
    w = net_weight if net_weight is not None else getattr(db, "net_weight", None)
    return None if w is None else np.ascontiguousarray(w, np.float32)


class QuadraticPlacer:
    """IInitialPlacer "init" (src/init/initial_placer.h:24-38)."""

    def __init__(self, params: QpParams | None = None):
        self.params = params or default_params()

    def place(self, db: PlaceDB, net_weight=None) -> dict:
        view = db.view()
        w = _weights(db, net_weight)
        x, y = db.node_x, db.node_y  # contiguous float32 after view()
        cap = max(1, int(self.params.max_iter))
        rows = (QpRow * cap)()
        n = C.c_int32(0)
        _check(_bind().spg_qp_place(C.byref(view), None if w is None else w.ctypes.data, C.byref(self.params),
                                    abi.fptr(x), abi.fptr(y), rows, cap, C.byref(n)))
        out = {f: np.array([getattr(rows[i], f) for i in range(n.value)]) for f, _ in QpRow._fields_}
        return out


def assemble(db: PlaceDB, axis: int, x=None, y=None, params: QpParams | None = None, net_weight=None):
    """The linear system of one axis at positions x, y: (row_start, col, val, rhs)."""
    p = params or default_params()
    view = db.view()
    x = np.ascontiguousarray(db.node_x if x is None else x, np.float32)
    y = np.ascontiguousarray(db.node_y if y is None else y, np.float32)
    w = _weights(db, net_weight)
    L = _bind()
    nnz = C.c_int64(0)
    wp = None if w is None else w.ctypes.data
    _check(L.spg_qp_assemble(C.byref(view), wp, C.byref(p), axis, abi.fptr(x), abi.fptr(y), None, None, None,
                             None, 0, C.byref(nnz)))
    n = db.num_movable
    start, col = np.zeros(n + 1, np.int32), np.zeros(nnz.value, np.int32)
    val, rhs = np.zeros(nnz.value, np.float32), np.zeros(n, np.float32)
    _check(L.spg_qp_assemble(C.byref(view), wp, C.byref(p), axis, abi.fptr(x), abi.fptr(y), abi.iptr(start),
                             abi.iptr(col), abi.fptr(val), abi.fptr(rhs), nnz.value, C.byref(nnz)))
    return start, col, val, rhs


def host_hpwl(db: PlaceDB, x=None, y=None) -> float:
    view = db.view()
    x = np.ascontiguousarray(db.node_x if x is None else x, np.float32)
    y = np.ascontiguousarray(db.node_y if y is None else y, np.float32)
    out = C.c_double()
    _check(_bind().spg_host_hpwl(C.byref(view), abi.fptr(x), abi.fptr(y), C.byref(out)))
    return out.value
