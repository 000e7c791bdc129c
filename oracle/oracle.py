"""ctypes access to oracle/liboracle.so, the C restatement of the GP operators.

TEST INFRASTRUCTURE: the checker of the CUDA path (tests/, smoke check, CPU-baseline leg
of bench.py). The product never imports this module.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from superplace_b200 import abi

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "liboracle.so")
_lib = None


class Grid(C.Structure):
    _fields_ = [("dim", C.c_int), ("step_x", C.c_float), ("step_y", C.c_float),
                ("origin_x", C.c_float), ("origin_y", C.c_float),
                ("target_density", C.c_float), ("movable_area_scaled", C.c_double)]


def lib():
    global _lib
    if _lib is None:
        L = C.CDLL(LIB_PATH)
        V = C.POINTER(abi.DbView)
        G = C.POINTER(Grid)
        fp, dp, ip = C.POINTER(C.c_float), C.POINTER(C.c_double), C.POINTER(C.c_int)
        i64p = C.POINTER(C.c_int64)
        L.spo_grid_setup.argtypes = [V, C.c_float, C.c_int, G]
        L.spo_static_density.argtypes = [V, G, fp, fp]
        L.spo_accumulate_chunks.argtypes = [V, G, C.c_int, fp, fp]
        L.spo_accumulate_fixed.argtypes = [V, G, C.c_int, i64p, i64p]
        L.spo_fixed_shift.argtypes = [V, G]
        L.spo_overflow.restype = C.c_float
        L.spo_overflow.argtypes = [G, fp, fp, fp]
        L.spo_rho.argtypes = [G, fp, fp, fp, fp, fp]
        L.spo_poisson_f64.argtypes = [C.c_int, C.c_int, C.c_double, C.c_double, dp, dp, dp, dp]
        L.spo_poisson.argtypes = [C.c_int, C.c_int, C.c_float, C.c_float, fp, fp, fp, fp]
        L.spo_gather.argtypes = [V, G, fp, fp, fp]
        L.spo_total_charge.restype = C.c_double
        L.spo_total_charge.argtypes = [V, G]
        L.spo_gamma.restype = C.c_float
        L.spo_gamma.argtypes = [C.c_float, C.c_float]
        L.spo_lambda_mu.restype = C.c_float
        L.spo_lambda_mu.argtypes = [C.c_double, C.c_double]
        L.spo_wa.restype = C.c_double
        L.spo_wa.argtypes = [V, C.c_float, C.c_int, fp]
        L.spo_hpwl.restype = C.c_double
        L.spo_hpwl.argtypes = [V]
        L.spo_chunk_sum.restype = C.c_double
        L.spo_chunk_sum.argtypes = [fp, C.c_int64, C.c_int]
        _lib = L
    return _lib


class OracleGrid:
    """BinGrid semantics over one PlaceDB (dimension, static terms, operators)."""

    def __init__(self, db, target_density=1.0, bin_dim=0):
        self.db = db
        self.view = db.view()
        self.g = Grid()
        lib().spo_grid_setup(C.byref(self.view), target_density, bin_dim, C.byref(self.g))
        d = self.g.dim
        self.terminal = np.zeros(d * d, np.float32)
        self.base = np.zeros(d * d, np.float32)
        lib().spo_static_density(C.byref(self.view), C.byref(self.g), abi.fptr(self.terminal),
                                 abi.fptr(self.base))

    @property
    def dim(self):
        return self.g.dim

    def refresh(self):
        """Re-take the view after the db arrays were replaced."""
        self.view = self.db.view()

    def accumulate_chunks(self, chunks=8):
        d = self.dim
        node, filler = np.zeros(d * d, np.float32), np.zeros(d * d, np.float32)
        lib().spo_accumulate_chunks(C.byref(self.view), C.byref(self.g), chunks, abi.fptr(node),
                                    abi.fptr(filler))
        return node, filler

    def fixed_shift(self):
        return lib().spo_fixed_shift(C.byref(self.view), C.byref(self.g))

    def accumulate_fixed(self, shift=None):
        d = self.dim
        if shift is None:
            shift = self.fixed_shift()
        node, filler = np.zeros(d * d, np.int64), np.zeros(d * d, np.int64)
        lib().spo_accumulate_fixed(C.byref(self.view), C.byref(self.g), shift,
                                   node.ctypes.data_as(C.POINTER(C.c_int64)),
                                   filler.ctypes.data_as(C.POINTER(C.c_int64)))
        return node, filler, shift

    def overflow(self, node):
        node = np.ascontiguousarray(node, np.float32).ravel()
        return lib().spo_overflow(C.byref(self.g), abi.fptr(node), abi.fptr(self.terminal),
                                  abi.fptr(self.base))

    def rho(self, node, filler):
        out = np.zeros(self.dim * self.dim, np.float32)
        node = np.ascontiguousarray(node, np.float32).ravel()
        filler = np.ascontiguousarray(filler, np.float32).ravel()
        lib().spo_rho(C.byref(self.g), abi.fptr(node), abi.fptr(filler), abi.fptr(self.terminal),
                      abi.fptr(self.base), abi.fptr(out))
        return out

    def gather(self, fx, fy):
        total = self.db.total_nodes
        out = np.zeros(2 * total, np.float32)
        fx = np.ascontiguousarray(fx, np.float32).ravel()
        fy = np.ascontiguousarray(fy, np.float32).ravel()
        lib().spo_gather(C.byref(self.view), C.byref(self.g), abi.fptr(fx), abi.fptr(fy),
                         abi.fptr(out))
        return out

    def total_charge(self):
        return lib().spo_total_charge(C.byref(self.view), C.byref(self.g))


def fixed_to_float(m, shift):
    """Fixed-point map -> float map exactly as the engine converts it (int64 -> double,
    times 2^-shift, rounded to float)."""
    return (m.astype(np.float64) * np.ldexp(1.0, -shift)).astype(np.float32)


def poisson_f64(rho, step_x, step_y):
    rho = np.ascontiguousarray(rho, np.float64)
    nx, ny = rho.shape
    out = [np.zeros_like(rho) for _ in range(3)]
    dp = C.POINTER(C.c_double)
    lib().spo_poisson_f64(nx, ny, step_x, step_y, rho.ctypes.data_as(dp),
                          *[o.ctypes.data_as(dp) for o in out])
    return tuple(out)


def wa(db, gamma, ignore=100):
    v = db.view()
    g = np.zeros(2 * db.num_movable, np.float32)
    wl = lib().spo_wa(C.byref(v), gamma, ignore, abi.fptr(g))
    return wl, g


def hpwl(db):
    v = db.view()
    return lib().spo_hpwl(C.byref(v))


def gamma(tau, step):
    return lib().spo_gamma(tau, step)


def lambda_mu(dh, ref):
    return lib().spo_lambda_mu(dh, ref)


def chunk_sum(a, mode=0):
    a = np.ascontiguousarray(a, np.float32)
    return lib().spo_chunk_sum(abi.fptr(a), a.size, mode)
