"""ctypes access to oracle/_ref/libspref.so: the reference's OWN CPU code for the GP path
(built from its sources by oracle/Makefile). Test infrastructure: only tests/, the smoke
check and the CPU-baseline leg of bench.py use it.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from superplace_b200 import abi

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_ref", "libspref.so")
_lib = None


def available() -> bool:
    return os.path.exists(LIB_PATH)


def lib():
    global _lib
    if _lib is None:
        L = C.CDLL(LIB_PATH)
        vp, fp, dp, ip = C.c_void_p, C.POINTER(C.c_float), C.POINTER(C.c_double), C.POINTER(C.c_int)
        L.spref_last_error.restype = C.c_char_p
        L.spref_db_create.restype = vp
        L.spref_db_create.argtypes = [C.POINTER(abi.DbView)]
        L.spref_db_destroy.argtypes = [vp]
        L.spref_db_counts.argtypes = [vp, ip]
        L.spref_db_regions.argtypes = [vp, fp, dp]
        L.spref_db_get_nodes.argtypes = [vp, fp, fp, fp, fp, C.POINTER(C.c_uint8)]
        L.spref_db_set_xy.argtypes = [vp, fp, fp]
        L.spref_db_set_flags.argtypes = [vp, C.POINTER(C.c_uint8)]
        L.spref_fillers_init.argtypes = [vp, C.c_float, C.c_uint64, dp]
        L.spref_fillers_scatter.argtypes = [vp, C.c_uint64, C.c_uint64]
        L.spref_grid_create.restype = vp
        L.spref_grid_create.argtypes = [vp, C.c_float, C.c_int, C.c_int]
        L.spref_grid_destroy.argtypes = [vp]
        L.spref_grid_info.argtypes = [vp, fp, dp]
        L.spref_grid_accumulate.argtypes = [vp, vp]
        L.spref_grid_overflow.restype = C.c_float
        L.spref_grid_overflow.argtypes = [vp]
        L.spref_grid_solve.argtypes = [vp]
        L.spref_grid_gather.argtypes = [vp, vp, fp]
        L.spref_grid_total_charge.restype = C.c_double
        L.spref_grid_total_charge.argtypes = [vp, vp]
        L.spref_grid_read.argtypes = [vp, C.c_int, fp]
        L.spref_wa.restype = C.c_double
        L.spref_wa.argtypes = [vp, C.c_float, C.c_int, fp]
        L.spref_hpwl.restype = C.c_double
        L.spref_hpwl.argtypes = [vp]
        L.spref_gamma.restype = C.c_float
        L.spref_gamma.argtypes = [C.c_float, C.c_float]
        L.spref_poisson.argtypes = [C.c_int, C.c_int, C.c_float, C.c_float, fp, fp, fp, fp]
        L.spref_poisson_bench.restype = C.c_double
        L.spref_poisson_bench.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int, fp]
        L.spref_eplace_run.argtypes = [vp, C.POINTER(abi.Params), C.c_int, dp, dp, dp, C.c_int, ip]
        L.spref_nesterov_quadratic.argtypes = [C.c_int, fp, fp, fp, C.c_int, C.c_int, C.c_int,
                                               C.c_float, dp]
        L.spref_set_threads.argtypes = [C.c_int]
        L.spref_max_threads.restype = C.c_int
        L.spref_quiet.argtypes = [C.c_int]
        L.spref_bookshelf_read.restype = vp
        L.spref_bookshelf_read.argtypes = [C.c_char_p]
        L.spref_db_more_counts.argtypes = [vp, C.POINTER(C.c_longlong)]
        L.spref_db_get_pins.argtypes = [vp, fp, fp, ip, ip, ip, ip, ip, ip]
        L.spref_db_get_rows.argtypes = [vp, fp, fp, fp, fp, ip]
        L.spref_db_get_names.argtypes = [vp, vp, vp, C.POINTER(C.c_uint8), fp]
        L.spref_write_pl.argtypes = [vp, C.c_char_p]
        L.spref_read_placement.argtypes = [vp, C.c_char_p]
        L.spref_abacus.argtypes = [vp, C.c_int, C.c_int, dp]
        L.spref_obj_and_grad.argtypes = [vp, C.POINTER(abi.Params), C.c_int, C.c_float, C.c_float, fp, fp, dp, ip]
        L.spref_legalize_macros.argtypes = [vp, C.POINTER(abi.Params), dp]
        L.spref_gp_four_stage.argtypes = [vp, C.POINTER(abi.Params), dp]
        L.spref_eplace_run_diagnostics.argtypes = [vp, C.POINTER(abi.Params), C.c_int, C.c_char_p, dp]
        L.spref_diagnose_delivered.argtypes = [vp, C.POINTER(abi.Params), C.c_int, C.c_char_p, C.c_int, C.c_float,
                                               C.c_float, C.c_int, fp, C.c_int]
        L.spref_quiet(1)
        _lib = L
    return _lib


def _f(a):
    return np.ascontiguousarray(a, np.float32)


class RefDb:
    """A reference sp::PlaceDB built from a superplace_b200 PlaceDB."""

    def __init__(self, db):
        self._view = db.view()
        self.h = lib().spref_db_create(C.byref(self._view))
        if not self.h:
            raise RuntimeError(lib().spref_last_error().decode())

    def __del__(self):
        if getattr(self, "h", None):
            lib().spref_db_destroy(self.h)
            self.h = None

    def counts(self):
        c = (C.c_int * 5)()
        lib().spref_db_counts(self.h, c)
        return tuple(c)

    def nodes(self):
        total = self.counts()[1] + self.counts()[2]
        x, y, w, h = (np.zeros(total, np.float32) for _ in range(4))
        f = np.zeros(total, np.uint8)
        lib().spref_db_get_nodes(self.h, abi.fptr(x), abi.fptr(y), abi.fptr(w), abi.fptr(h),
                                 abi.u8ptr(f))
        return x, y, w, h, f

    def set_xy(self, x, y):
        x, y = _f(x), _f(y)
        lib().spref_db_set_xy(self.h, abi.fptr(x), abi.fptr(y))

    def set_flags(self, flags):
        f = np.ascontiguousarray(flags, np.uint8)
        lib().spref_db_set_flags(self.h, abi.u8ptr(f))

    def fillers_init(self, target_density=1.0, seed=1002):
        info = (C.c_double * 6)()
        rc = lib().spref_fillers_init(self.h, target_density, seed, info)
        if rc:
            raise RuntimeError(lib().spref_last_error().decode())
        return list(info)

    def hpwl(self):
        return lib().spref_hpwl(self.h)

    def wa(self, gamma, ignore=100):
        n = self.counts()[0]
        g = np.zeros(2 * n, np.float32)
        wl = lib().spref_wa(self.h, gamma, ignore, abi.fptr(g))
        return wl, g

    def eplace(self, params, stage=abi.STAGE_MGP, cap=4000):
        """EPlace(db, cfg, sink).run(stage): the result dict and the stage's metrics rows, one
        row of ROW_FIELDS per iteration."""
        res = (C.c_double * 8)()
        init = (C.c_double * 3)()
        rows = np.zeros((cap, len(ROW_FIELDS)), np.float64)
        nrows = C.c_int(0)
        rc = lib().spref_eplace_run(self.h, C.byref(params), stage, res, init,
                                    rows.ctypes.data_as(C.POINTER(C.c_double)), cap,
                                    C.byref(nrows))
        if rc:
            raise RuntimeError(f"{rc}: " + lib().spref_last_error().decode())
        return dict(zip(RESULT_FIELDS, list(res))), rows[: nrows.value]

    def eplace_diagnostics(self, params, root, stage=abi.STAGE_MGP):
        """EPlace::run with gp_diagnostics on, its sink writing under root: the reference's own GP
        diagnostics of the stage; returns the result dict."""
        res = (C.c_double * 8)()
        rc = lib().spref_eplace_run_diagnostics(self.h, C.byref(params), stage, str(root).encode(), res)
        if rc:
            raise RuntimeError(f"{rc}: " + lib().spref_last_error().decode())
        return dict(zip(RESULT_FIELDS, list(res)))

    def diagnose_delivered(self, params, root, stage, it, lam, gamma, dim, previous=None):
        """diagnoseDelivered (src/gp/diagnostics.cpp:175-191) at the handle's positions."""
        prev = _f(previous) if previous is not None else None
        rc = lib().spref_diagnose_delivered(self.h, C.byref(params), stage, str(root).encode(), int(it), float(lam),
                                            float(gamma), int(dim), prev.ctypes.data_as(C.POINTER(C.c_float))
                                            if prev is not None else None, 0 if prev is None else prev.size)
        if rc:
            raise RuntimeError(f"{rc}: " + lib().spref_last_error().decode())

    def n_opt(self, params, stage=abi.STAGE_MGP):
        n = C.c_int(0)
        lib().spref_obj_and_grad(self.h, C.byref(params), stage, 1.0, 1.0, None, None, None, C.byref(n))
        return n.value

    def obj_and_grad(self, params, stage, lam, gamma, pos):
        """EPlace::Impl::objAndGrad (src/gp/eplace.cpp:136-203) at opt-set positions pos (x then
        y), composed from the reference's operators: (grad, {obj, tau, hpwl, sum_wl, sum_den})."""
        pos = _f(pos)
        grad = np.zeros_like(pos)
        out = (C.c_double * 5)()
        n = C.c_int(0)
        if lib().spref_obj_and_grad(self.h, C.byref(params), stage, lam, gamma, abi.fptr(pos), abi.fptr(grad),
                                    out, C.byref(n)):
            raise RuntimeError(lib().spref_last_error().decode())
        return grad, dict(zip(("obj", "tau", "hpwl", "sum_wl", "sum_den"), list(out)))

    def legalize_macros(self, params):
        """legalizeMacros (src/lg/macro_sa.cpp:493) in place; the macros end F_FIXED."""
        res = (C.c_double * 6)()
        if lib().spref_legalize_macros(self.h, C.byref(params), res):
            raise RuntimeError(lib().spref_last_error().decode())
        return dict(zip(MLG_FIELDS, list(res)))

    def gp_four_stage(self, params):
        """GlobalPlaceStage's sequence for movable macros (src/stages/gp_stage.cpp:99-201): mGP,
        mLG, scatterFillers(seed offset 1), FILLERONLY, cGP. Per stage its result dict, and mLG's."""
        res = (C.c_double * 30)()
        if lib().spref_gp_four_stage(self.h, C.byref(params), res):
            raise RuntimeError(lib().spref_last_error().decode())
        out = {name: dict(zip(RESULT_FIELDS, list(res)[8 * k: 8 * k + 8]))
               for k, name in enumerate(("mGP", "FILLERONLY", "cGP"))}
        out["mLG"] = dict(zip(MLG_FIELDS, list(res)[24:30]))
        return out


RESULT_FIELDS = ("iterations", "hpwl", "overflow", "converged", "stagnated", "rollback_iter",
                 "evaluations", "elapsed_ms")
# sp::IterMetrics (src/util/metrics.h:12-28) as the shim writes it
ROW_FIELDS = ("iter", "hpwl", "overflow", "lambda", "gamma", "step_size", "evaluations", "elapsed_ms",
              "grad_norm_wl", "grad_norm_den", "eval_lambda", "eval_gamma", "delta_hpwl", "lambda_mu")
MLG_FIELDS = ("num_macros", "overlap_before", "overlap_after", "hpwl_before", "hpwl_after", "repaired")


def bookshelf_read(aux_path):
    """The reference's BookshelfReader::read (src/io/bookshelf_reader.cpp:433-463) into a RefDb."""
    h = lib().spref_bookshelf_read(os.fsencode(aux_path))
    if not h:
        raise RuntimeError(lib().spref_last_error().decode())
    r = RefDb.__new__(RefDb)
    r.h = h
    return r


def bookshelf_arrays(r: RefDb) -> dict:
    """Every array of a reference PlaceDB that BookShelf reading fills, keyed like PlaceDB."""
    num_movable, num_nodes, _, num_pins, num_nets = r.counts()
    more = (C.c_longlong * 3)()
    lib().spref_db_more_counts(r.h, more)
    num_rows, node_bytes, net_bytes = (int(v) for v in more)
    x, y, w, h, flags = r.nodes()
    out = dict(num_movable=num_movable, num_nodes=num_nodes, node_x=x, node_y=y, node_w=w, node_h=h,
               node_flags=flags)
    f32 = lambda n: np.zeros(n, np.float32)  # noqa: E731
    i32 = lambda n: np.zeros(n, np.int32)  # noqa: E731
    ox, oy = f32(num_pins), f32(num_pins)
    p2n, p2net, fn2p, fnd2p = (i32(num_pins) for _ in range(4))
    n2ps, nd2ps = i32(num_nets + 1), i32(num_nodes + 1)
    lib().spref_db_get_pins(r.h, abi.fptr(ox), abi.fptr(oy), abi.iptr(p2n), abi.iptr(p2net), abi.iptr(n2ps),
                            abi.iptr(fn2p), abi.iptr(nd2ps), abi.iptr(fnd2p))
    out.update(pin_offset_x=ox, pin_offset_y=oy, pin2node=p2n, pin2net=p2net, net2pin_start=n2ps,
               flat_net2pin=fn2p, node2pin_start=nd2ps, flat_node2pin=fnd2p)
    ly, hh, lx, st = (f32(num_rows) for _ in range(4))
    sites = i32(num_rows)
    lib().spref_db_get_rows(r.h, abi.fptr(ly), abi.fptr(hh), abi.fptr(lx), abi.fptr(st), abi.iptr(sites))
    out.update(row_ly=ly, row_height=hh, row_lx=lx, row_step=st, row_num_sites=sites)
    nn, tn = np.zeros(max(node_bytes, 1), np.uint8), np.zeros(max(net_bytes, 1), np.uint8)
    orient, weight = np.zeros(num_nodes, np.uint8), f32(num_nets)
    lib().spref_db_get_names(r.h, nn.ctypes.data, tn.ctypes.data, abi.u8ptr(orient), abi.fptr(weight))
    out.update(node_orient=orient, net_weight=weight,
               node_names=[s.decode() for s in bytes(nn).split(b"\0")[:num_nodes]],
               net_names=[s.decode() for s in bytes(tn).split(b"\0")[:num_nets]])
    core = (C.c_float * 5)()
    area = C.c_double()
    lib().spref_db_regions(r.h, core, C.byref(area))
    out.update(core=tuple(core[:4]), row_height_mode=core[4], total_row_area=area.value)
    return out


ABACUS_FIELDS = ("precondition_ok", "cells", "failed", "rows", "segments", "rounded_widths",
                 "selfcheck_overlaps", "selfcheck_off_site", "disp_mean", "disp_max")


def abacus(r: RefDb, area_weight=False, reference_trials=False) -> dict:
    """The reference's legalizeCells (src/lg/abacus.cpp:155-284) on the RefDb, in place."""
    res = (C.c_double * 10)()
    if lib().spref_abacus(r.h, int(area_weight), int(reference_trials), res):
        raise ValueError(lib().spref_last_error().decode())
    return {k: (res[i] if i >= 8 else int(res[i])) for i, k in enumerate(ABACUS_FIELDS)}


CHECK_PATH = os.path.join(_HERE, "_ref", "superplace-check")


def check_placement(aux, pl=None):
    """The reference's legality checker (tools/check/main.cpp, built by oracle/Makefile) on a
    design and a placement: (exit code, report text). 0 = PASS, 1 = FAIL, 2 = bad input."""
    import subprocess
    args = [CHECK_PATH, str(aux)] + ([str(pl)] if pl else [])
    out = subprocess.run(args, capture_output=True, text=True, timeout=600)
    return out.returncode, out.stdout


def read_placement(r: RefDb, path):
    """The reference's BookshelfReader::readPlacement (src/io/bookshelf_reader.cpp:367-401)."""
    if lib().spref_read_placement(r.h, os.fsencode(path)):
        raise RuntimeError(lib().spref_last_error().decode())


def write_pl(r: RefDb, path):
    """The reference's BookshelfWriter::writePl (src/io/bookshelf_writer.cpp:16-37)."""
    if lib().spref_write_pl(r.h, os.fsencode(path)):
        raise RuntimeError(lib().spref_last_error().decode())


class RefGrid:
    def __init__(self, rdb: RefDb, target_density=1.0, bin_dim=0, chunks=0):
        self.rdb = rdb
        self.h = lib().spref_grid_create(rdb.h, target_density, bin_dim, chunks)
        if not self.h:
            raise RuntimeError(lib().spref_last_error().decode())
        info = (C.c_float * 5)()
        den = C.c_double()
        lib().spref_grid_info(self.h, info, C.byref(den))
        self.dim = int(info[0])
        self.step_x, self.step_y, self.origin_x, self.origin_y = info[1], info[2], info[3], info[4]
        self.overflow_denominator = den.value

    def __del__(self):
        if getattr(self, "h", None):
            lib().spref_grid_destroy(self.h)
            self.h = None

    def accumulate(self):
        lib().spref_grid_accumulate(self.h, self.rdb.h)

    def overflow(self):
        return lib().spref_grid_overflow(self.h)

    def solve(self):
        lib().spref_grid_solve(self.h)

    def gather(self):
        total = self.rdb.counts()[1] + self.rdb.counts()[2]
        f = np.zeros(2 * total, np.float32)
        lib().spref_grid_gather(self.h, self.rdb.h, abi.fptr(f))
        return f

    def total_charge(self):
        return lib().spref_grid_total_charge(self.h, self.rdb.h)

    def read(self, which):
        out = np.zeros(self.dim * self.dim, np.float32)
        lib().spref_grid_read(self.h, which, abi.fptr(out))
        return out.reshape(self.dim, self.dim)


def poisson(rho, step_x, step_y):
    rho = _f(rho)
    nx, ny = rho.shape
    phi, ex, ey = (np.zeros_like(rho) for _ in range(3))
    rc = lib().spref_poisson(nx, ny, step_x, step_y, abi.fptr(rho), abi.fptr(phi),
                             abi.fptr(ex), abi.fptr(ey))
    if rc:
        raise RuntimeError(lib().spref_last_error().decode())
    return phi, ex, ey


def gamma(tau, step):
    return lib().spref_gamma(tau, step)


def nesterov_quadratic(coef, target, pos, steps, use_bb=True, backtrack=False, init_step=0.0):
    coef, target = _f(coef), _f(target)
    pos = _f(pos).copy()
    out = (C.c_double * 3)()
    rc = lib().spref_nesterov_quadratic(pos.size, abi.fptr(coef), abi.fptr(target), abi.fptr(pos),
                                        steps, int(use_bb), int(backtrack), init_step, out)
    if rc:
        raise RuntimeError(lib().spref_last_error().decode())
    return pos, out[0], int(out[1]), out[2]
