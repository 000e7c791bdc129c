"""The init stage's placers by name, as makeInitialPlacer (src/init/initial_placer.cpp:9-23) offers
them: "random", "cluster_fc", "cluster_bc" (spg_random_place / spg_cluster_place, host code) and
"quadratic" (superplace_b200.qp, the default init_method). Each moves the PlaceDB's movable
nodes in place.
"""
from __future__ import annotations

import ctypes as C

from . import abi, qp
from .engine import SpgError, lib
from .placedb import PlaceDB

METHODS = ("random", "cluster_fc", "cluster_bc", "quadratic")


def _bind():
    L = lib()
    if not getattr(L, "_init_bound", False):
        fp, ip = C.POINTER(C.c_float), C.POINTER(C.c_int32)
        L.spg_init_last_error.restype = C.c_char_p
        L.spg_random_place.argtypes = [C.POINTER(abi.DbView), C.c_uint64, fp, fp]
        L.spg_cluster_place.argtypes = [C.POINTER(abi.DbView), C.c_int32, C.c_int32, C.c_int32, fp, fp, ip, ip]
        L._init_bound = True
    return L


def _check(rc):
    if rc != 0:
        raise SpgError(rc, _bind().spg_init_last_error().decode())


class InitialPlacer:
    """IInitialPlacer (src/init/initial_placer.h:24-38): place(db) returns a small report."""

    def __init__(self, method: str = "quadratic", seed: int = 1002, cluster_target_count: int = 0,
                 ignore_net_degree: int = 100, qp_params=None):
        if method not in METHODS:
            raise ValueError(f"unknown init method {method!r}; one of {METHODS}")
        self.method, self.seed = method, seed
        self.target, self.ignore = cluster_target_count, ignore_net_degree
        self.qp_params = qp_params

    def place(self, db: PlaceDB) -> dict:
        if self.method == "quadratic":
            rows = qp.QuadraticPlacer(self.qp_params).place(db)
            return {"method": self.method, "outer_iters": int(rows["iter"].shape[0])}
        view = db.view()
        L = _bind()
        if self.method == "random":
            _check(L.spg_random_place(C.byref(view), self.seed, abi.fptr(db.node_x), abi.fptr(db.node_y)))
            return {"method": self.method}
        clusters, levels = C.c_int32(0), C.c_int32(0)
        _check(L.spg_cluster_place(C.byref(view), int(self.method == "cluster_bc"), self.target, self.ignore,
                                   abi.fptr(db.node_x), abi.fptr(db.node_y), C.byref(clusters), C.byref(levels)))
        return {"method": self.method, "clusters": clusters.value, "levels": levels.value}


def make_initial_placer(method: str, **kw) -> InitialPlacer:
    return InitialPlacer(method, **kw)
