"""Python host over the C ABI (include/spgpu.h), mirroring the reference's operator API
for the GP path:

* ``make_poisson_backend`` / ``PoissonBackend.solve``  — src/numeric/poisson_backend.h:20-60
* ``initialize_fillers`` / ``scatter_fillers``        — src/gp/filler.h:29-32
* ``BinGrid``-style operators on ``GpContext``        — src/gp/bin_grid.h:23-52
* ``GpContext.wa`` / ``GpContext.hpwl``               — src/gp/wa_wirelength.h:29-33, src/db/hpwl.h:16
* ``EPlace.run``                                      — src/gp/eplace.h:56-77

There is no CPU fallback: if libspgpu.so is missing or no sm_100 device is visible, the
constructors raise.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from . import abi
from .placedb import PlaceDB

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libspgpu.so")
_lib = None
# spg_iter_fn: (user, stage, iter, x, y)
ITER_FN = C.CFUNCTYPE(None, C.c_void_p, C.c_int32, C.c_int32, C.POINTER(C.c_float), C.POINTER(C.c_float))


class SpgError(RuntimeError):
    """A failed C-ABI call; ``kind`` is the reference InvariantError kind when it maps to one."""

    def __init__(self, code, msg):
        super().__init__(f"[{code}] {msg}")
        self.code = code
        self.kind = abi.ERROR_KINDS.get(code)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is not built (run python -m superplace_b200.build)")
        L = C.CDLL(LIB_PATH)
        vp, fp, dp, ip = C.c_void_p, C.POINTER(C.c_float), C.POINTER(C.c_double), C.POINTER(C.c_int)
        i64p = C.POINTER(C.c_int64)
        L.spg_last_error.restype = C.c_char_p
        L.spg_poisson_name.restype = C.c_char_p
        L.spg_poisson_name.argtypes = [vp]
        L.spg_poisson_create_batched.argtypes = [C.c_int, C.c_int, C.c_float, C.c_float, C.c_int,
                                                 C.c_int, C.POINTER(vp)]
        L.spg_poisson_create.argtypes = [C.c_int, C.c_int, C.c_float, C.c_float, C.c_int,
                                         C.POINTER(vp)]
        L.spg_poisson_solve.argtypes = [vp, fp, fp, fp, fp]
        L.spg_poisson_solve_device.argtypes = [vp, vp, vp, vp, vp, vp]
        L.spg_poisson_solve_batch_device.argtypes = [vp, C.c_int, vp, vp, vp, vp, vp]
        L.spg_poisson_destroy.argtypes = [vp]
        L.spg_poisson_set_single_launch.argtypes = [vp, C.c_int]
        L.spg_poisson_solve_static.argtypes = [C.c_int, C.c_int, C.c_float, C.c_float, vp, vp, vp,
                                               vp, vp]
        L.spg_fillers_plan.argtypes = [C.POINTER(abi.DbView), C.c_float, C.POINTER(abi.FillerInfo)]
        L.spg_fillers_scatter.argtypes = [C.POINTER(abi.DbView), C.c_int32, C.c_float, C.c_float,
                                          C.c_uint64, fp, fp]
        L.spg_ctx_create.argtypes = [C.POINTER(abi.DbView), C.POINTER(abi.Params), C.POINTER(vp)]
        L.spg_ctx_destroy.argtypes = [vp]
        L.spg_ctx_load.argtypes = [vp, C.POINTER(abi.DbView), C.POINTER(abi.Params)]
        L.spg_positions_h2d.argtypes = [vp, fp, fp]
        L.spg_positions_d2h.argtypes = [vp, fp, fp]
        L.spg_flags_h2d.argtypes = [vp, C.POINTER(C.c_uint8)]
        L.spg_host_alloc.argtypes = [C.c_size_t, C.POINTER(vp)]
        L.spg_set_iter_callback.argtypes = [vp, ITER_FN, vp, C.c_int32]
        L.spg_eval_positions.argtypes = [vp, C.c_int32, fp, fp]
        L.spg_set_stagnation_callback.argtypes = [vp, ITER_FN, vp]
        L.spg_host_free.argtypes = [vp]
        L.spg_grid_init.argtypes = [vp, C.c_float, C.c_int]
        L.spg_grid_info.argtypes = [vp, ip, fp, fp, fp, fp, dp]
        L.spg_grid_read.argtypes = [vp, C.c_int, fp]
        L.spg_grid_write.argtypes = [vp, C.c_int, fp]
        L.spg_grid_read_fixed.argtypes = [vp, i64p, i64p, ip]
        L.spg_density_accumulate.argtypes = [vp]
        L.spg_overflow.argtypes = [vp, fp]
        L.spg_solve_field.argtypes = [vp]
        L.spg_gather_force.argtypes = [vp, fp]
        L.spg_total_charge.argtypes = [vp, dp]
        L.spg_wa_wirelength.argtypes = [vp, C.c_float, C.c_int, dp, fp]
        L.spg_hpwl.argtypes = [vp, dp]
        L.spg_stage_run.argtypes = [vp, C.c_int, C.POINTER(abi.Result)]
        L.spg_metrics_d2h.argtypes = [vp, C.POINTER(abi.IterMetrics), C.c_int, ip]
        L.spg_ctx_launch_count.restype = C.c_int64
        L.spg_ctx_launch_count.argtypes = [vp]
        L.spg_ctx_stream.restype = vp
        L.spg_ctx_stream.argtypes = [vp]
        L.spg_ctx_graph_loop.argtypes = [vp]
        L.spg_ctx_profile.argtypes = [vp, C.c_int, C.POINTER(C.c_double), C.c_int]
        L.spg_eval_grad.argtypes = [vp, C.c_int, C.c_float, C.c_float, fp, fp, dp, ip]
        L.spg_nesterov_quadratic.argtypes = [C.c_int32, fp, fp, fp, C.c_int32, C.c_int32, C.c_int32,
                                             C.c_int32, C.c_float, dp]
        u8p, cp = C.POINTER(C.c_uint8), C.c_char_p
        L.spg_bookshelf_read.argtypes = [cp, C.POINTER(vp)]
        L.spg_bookshelf_last_error.restype = cp
        L.spg_bookshelf_counts.argtypes = [vp, i64p]
        L.spg_bookshelf_nodes.argtypes = [vp, fp, fp, fp, fp, u8p, u8p, vp]
        L.spg_bookshelf_pins.argtypes = [vp, fp, fp, ip, ip, ip, ip, ip, ip]
        L.spg_bookshelf_nets.argtypes = [vp, fp, vp]
        L.spg_bookshelf_rows.argtypes = [vp, fp, fp, fp, fp, ip]
        L.spg_bookshelf_destroy.argtypes = [vp]
        L.spg_bookshelf_write_pl.argtypes = [cp, C.c_int32, vp, fp, fp, fp, fp, u8p, u8p]
        L.spg_bookshelf_apply_pl.argtypes = [cp, C.c_int32, vp, fp, fp, fp, fp, u8p, u8p]
        _lib = L
    return _lib


def check(rc):
    if rc != 0:
        raise SpgError(rc, lib().spg_last_error().decode())


def device_available() -> bool:
    return lib().spg_device_check() == 0


def launch_count() -> int:
    return int(lib().spg_ctx_launch_count(None))


class _PinnedBlock:
    """Page-locked host memory from spg_host_alloc, freed with the last array viewing it."""

    def __init__(self, nbytes):
        self.ptr = C.c_void_p()
        check(lib().spg_host_alloc(max(int(nbytes), 1), C.byref(self.ptr)))
        self.nbytes = int(nbytes)
        self.__array_interface__ = {"shape": (self.nbytes,), "typestr": "|u1", "version": 3,
                                    "data": (self.ptr.value, False)}

    def __del__(self):
        if self.ptr:
            try:
                lib().spg_host_free(self.ptr)
            except Exception:  # interpreter shutdown: the process frees it
                pass
            self.ptr = C.c_void_p()


def pinned_empty(n, dtype) -> np.ndarray:
    """A 1-D array of n elements in page-locked host memory: the context's position copies
    from and into such arrays are direct DMA, with no staging copy on the host."""
    dtype = np.dtype(dtype)
    return np.asarray(_PinnedBlock(n * dtype.itemsize)).view(dtype)


def pin_positions(db: PlaceDB) -> PlaceDB:
    """Move the PlaceDB's node positions and flags into page-locked memory (values kept), so
    that EPlace.run's uploads and its read-back of the result are direct DMA."""
    for k, dt in (("node_x", np.float32), ("node_y", np.float32), ("node_flags", np.uint8)):
        a = np.ascontiguousarray(getattr(db, k), dt)
        p = pinned_empty(a.size, dt)
        p[:] = a
        setattr(db, k, p)
    return db


# ------------------------------------------------------------------ Poisson operator
class PoissonBackend:
    """PoissonBackend (src/numeric/poisson_backend.h:20-46) on the device.

    ``solve(density, phi, field_x, field_y)`` takes and fills host arrays of shape
    (nx, ny) (row-major, y fast), as the reference's spans."""

    def __init__(self, nx, ny, step_x, step_y, precision=abi.POISSON_FP32, batch=1, single_launch=False):
        self.nx, self.ny = int(nx), int(ny)
        h = C.c_void_p()
        check(lib().spg_poisson_create_batched(self.nx, self.ny, step_x, step_y, precision, batch,
                                               C.byref(h)))
        self.h = h
        if single_launch:  # one persistent launch per one-grid split-BF16 solve (spg_poisson_set_single_launch)
            check(lib().spg_poisson_set_single_launch(self.h, 1))

    def __del__(self):
        if getattr(self, "h", None) and _lib is not None:
            _lib.spg_poisson_destroy(self.h)
            self.h = None

    def name(self) -> str:
        return lib().spg_poisson_name(self.h).decode()

    def solve(self, density, phi=None, field_x=None, field_y=None):
        rho = np.ascontiguousarray(density, np.float32).reshape(self.nx, self.ny)
        phi = np.empty_like(rho) if phi is None else phi
        fx = np.empty_like(rho) if field_x is None else field_x
        fy = np.empty_like(rho) if field_y is None else field_y
        check(lib().spg_poisson_solve(self.h, abi.fptr(rho), abi.fptr(phi), abi.fptr(fx),
                                      abi.fptr(fy)))
        return phi, fx, fy

    def solve_device(self, rho_ptr, phi_ptr, fx_ptr, fy_ptr, stream=0, batch=1):
        """Device-pointer solve (ints are raw device addresses)."""
        check(lib().spg_poisson_solve_batch_device(self.h, batch, C.c_void_p(rho_ptr),
                                                   C.c_void_p(phi_ptr), C.c_void_p(fx_ptr),
                                                   C.c_void_p(fy_ptr), C.c_void_p(stream)))


def make_poisson_backend(nx, ny, step_x=1.0, step_y=1.0, precision=abi.POISSON_FP32):
    return PoissonBackend(nx, ny, step_x, step_y, precision)


def poisson_solve_static(nx, ny, step_x, step_y, rho_ptr, phi_ptr, fx_ptr, fy_ptr, stream=0):
    """spg_poisson_solve_static: the FP32 solve with no allocation at all (scratch in a
    static device array; nx, ny <= 512). Arguments are raw device addresses; for callers
    that cannot call cudaMalloc and so cannot build a PoissonBackend plan."""
    check(lib().spg_poisson_solve_static(int(nx), int(ny), step_x, step_y, C.c_void_p(rho_ptr),
                                         C.c_void_p(phi_ptr), C.c_void_p(fx_ptr),
                                         C.c_void_p(fy_ptr), C.c_void_p(stream)))


# ------------------------------------------------------------------ optimizer test hook
def nesterov_quadratic(coef, target, pos, steps, use_bb=True, backtrack=False, init_step=0.0, max_backtrack=10):
    """The stage loop's Nesterov optimizer on 0.5 * sum c (x - t)^2 (spg_nesterov_quadratic),
    `steps` calls of NesterovOptimizer::step: (v, objective, evaluations, step size, redos)."""
    coef = np.ascontiguousarray(coef, np.float32)
    target = np.ascontiguousarray(target, np.float32)
    pos = np.array(pos, np.float32)
    out = (C.c_double * 4)()
    check(lib().spg_nesterov_quadratic(pos.size, abi.fptr(coef), abi.fptr(target), abi.fptr(pos), steps,
                                       int(use_bb), int(backtrack), max_backtrack, init_step, out))
    return pos, out[0], int(out[1]), out[2], int(out[3])


# ------------------------------------------------------------------ fillers
def initialize_fillers(db: PlaceDB, target_density=1.0, seed=1002) -> abi.FillerInfo:
    """initializeFillers (src/gp/filler.cpp:47-139): replaces db's filler segment."""
    db.num_fillers = 0
    db.node_x, db.node_y = db.node_x[: db.num_nodes], db.node_y[: db.num_nodes]
    db.node_w, db.node_h = db.node_w[: db.num_nodes], db.node_h[: db.num_nodes]
    db.node_flags = db.node_flags[: db.num_nodes]
    db.extend_node2pin()
    v = db.view()
    info = abi.FillerInfo()
    check(lib().spg_fillers_plan(C.byref(v), target_density, C.byref(info)))
    if info.count > 0:
        x = np.zeros(info.count, np.float32)
        y = np.zeros(info.count, np.float32)
        check(lib().spg_fillers_scatter(C.byref(v), info.count, info.width, info.height, seed,
                                        abi.fptr(x), abi.fptr(y)))
        db.set_fillers(info.count, info.width, info.height, x, y)
    return info


def scatter_fillers(db: PlaceDB, seed=1002, seed_offset=0) -> None:
    """scatterFillers (src/gp/filler.cpp:33-45) for the existing fillers."""
    if db.num_fillers == 0:
        return
    v = db.view()
    x = np.zeros(db.num_fillers, np.float32)
    y = np.zeros(db.num_fillers, np.float32)
    w = float(db.node_w[db.num_nodes])
    h = float(db.node_h[db.num_nodes])
    check(lib().spg_fillers_scatter(C.byref(v), db.num_fillers, w, h, seed + seed_offset,
                                    abi.fptr(x), abi.fptr(y)))
    db.node_x[db.num_nodes:] = x
    db.node_y[db.num_nodes:] = y


# ------------------------------------------------------------------ placement context
MAP_NODE, MAP_FILLER, MAP_TERMINAL, MAP_BASE, MAP_RHO, MAP_PHI, MAP_XI_X, MAP_XI_Y = range(8)


class GpContext:
    """A PlaceDB resident on the device, with the BinGrid / WA / HPWL operators and the
    stage loop. Positions live on the device between calls."""

    def __init__(self, db: PlaceDB, params: abi.Params | None = None):
        self.db = db
        self.params = params or abi.default_params()
        self._view = db.view()
        h = C.c_void_p()
        check(lib().spg_ctx_create(C.byref(self._view), C.byref(self.params), C.byref(h)))
        self.h = h
        self.dim = 0

    def load(self, db: PlaceDB, params: abi.Params | None = None):
        """Replace the netlist (and parameters) with another instance, keeping the context's
        streams and device buffers (spg_ctx_load): what a placement server does per request."""
        self.db = db
        self.params = params or self.params
        self._view = db.view()
        check(lib().spg_ctx_load(self.h, C.byref(self._view), C.byref(self.params)))
        self.dim = 0

    def close(self):
        if getattr(self, "h", None) and _lib is not None:
            _lib.spg_ctx_destroy(self.h)
            self.h = None

    __del__ = close

    def graph_loop(self) -> bool:
        """Whether the last stage run executed its loop as one conditional CUDA graph."""
        return bool(lib().spg_ctx_graph_loop(self.h))

    PROFILE_PARTS = ("update", "wa", "scatter", "rho", "poisson", "assemble", "reduce", "evaluation")

    def profile(self, reps=20) -> dict:
        """Warm-L2 device time (us) of each iteration part at the current positions,
        CUDA events on the context's stream; the stage's results are left unchanged."""
        out = (C.c_double * 8)()
        check(lib().spg_ctx_profile(self.h, reps, out, 8))
        # "reduce" reports 0 (the norms and decisions run inside the assembly), and so does
        # "scatter" when every density node is in the opt set (the update scatters them)
        return {k: v for k, v in zip(self.PROFILE_PARTS, list(out)) if v > 0.0}

    def stream(self) -> int:
        """Raw cudaStream_t of this context (every call enqueues on it)."""
        return int(lib().spg_ctx_stream(self.h) or 0)

    # positions and flags
    def set_positions(self, x=None, y=None):
        x = np.ascontiguousarray(self.db.node_x if x is None else x, np.float32)
        y = np.ascontiguousarray(self.db.node_y if y is None else y, np.float32)
        check(lib().spg_positions_h2d(self.h, abi.fptr(x), abi.fptr(y)))

    def positions(self, out=None):
        """Node positions (x, y) from the device; into `out` = (x, y) when given (float32,
        contiguous, one entry per node), else into new arrays."""
        n = self.db.total_nodes
        if out is None:
            x, y = np.empty(n, np.float32), np.empty(n, np.float32)
        else:
            x, y = out
            for a in (x, y):
                if a.dtype != np.float32 or a.shape != (n,) or not a.flags.c_contiguous or not a.flags.writeable:
                    raise ValueError("positions(out=...): float32 contiguous writable arrays of one entry per node")
        check(lib().spg_positions_d2h(self.h, abi.fptr(x), abi.fptr(y)))
        return x, y

    def set_flags(self, flags):
        f = np.ascontiguousarray(flags, np.uint8)
        check(lib().spg_flags_h2d(self.h, abi.u8ptr(f)))

    # BinGrid
    def grid_init(self, target_density=None, bin_dim=None):
        td = self.params.target_density if target_density is None else target_density
        bd = self.params.gp_bin_dim if bin_dim is None else bin_dim
        check(lib().spg_grid_init(self.h, td, bd))
        info = self.grid_info()
        self.dim = info["dim"]
        return info

    def grid_info(self):
        d = C.c_int()
        sx, sy, ox, oy = C.c_float(), C.c_float(), C.c_float(), C.c_float()
        den = C.c_double()
        check(lib().spg_grid_info(self.h, C.byref(d), C.byref(sx), C.byref(sy), C.byref(ox),
                                  C.byref(oy), C.byref(den)))
        return dict(dim=d.value, step_x=sx.value, step_y=sy.value, origin_x=ox.value,
                    origin_y=oy.value, overflow_denominator=den.value)

    def read_map(self, which):
        out = np.zeros(self.dim * self.dim, np.float32)
        check(lib().spg_grid_read(self.h, which, abi.fptr(out)))
        return out.reshape(self.dim, self.dim)

    def write_map(self, which, a):
        a = np.ascontiguousarray(a, np.float32).ravel()
        check(lib().spg_grid_write(self.h, which, abi.fptr(a)))

    def read_fixed(self):
        n = self.dim * self.dim
        a, b = np.zeros(n, np.int64), np.zeros(n, np.int64)
        s = C.c_int()
        check(lib().spg_grid_read_fixed(self.h, a.ctypes.data_as(C.POINTER(C.c_int64)),
                                        b.ctypes.data_as(C.POINTER(C.c_int64)), C.byref(s)))
        return a, b, s.value

    def accumulate(self):
        check(lib().spg_density_accumulate(self.h))

    def overflow(self) -> float:
        t = C.c_float()
        check(lib().spg_overflow(self.h, C.byref(t)))
        return t.value

    def solve_field(self):
        check(lib().spg_solve_field(self.h))

    def gather_force(self):
        out = np.zeros(2 * self.db.total_nodes, np.float32)
        check(lib().spg_gather_force(self.h, abi.fptr(out)))
        return out

    def total_charge(self) -> float:
        c = C.c_double()
        check(lib().spg_total_charge(self.h, C.byref(c)))
        return c.value

    # wirelength
    def wa(self, gamma, ignore_net_degree=100):
        g = np.zeros(2 * self.db.num_movable, np.float32)
        wl = C.c_double()
        check(lib().spg_wa_wirelength(self.h, gamma, ignore_net_degree, C.byref(wl), abi.fptr(g)))
        return wl.value, g

    def hpwl(self) -> float:
        v = C.c_double()
        check(lib().spg_hpwl(self.h, C.byref(v)))
        return v.value

    def n_opt(self, stage=abi.STAGE_MGP) -> int:
        """Size of the stage's optimisation set (buildOptSet) at the context's flags."""
        n = C.c_int()
        check(lib().spg_eval_grad(self.h, stage, 1.0, 1.0, None, None, None, C.byref(n)))
        return n.value

    def eval_grad(self, stage, lam, gamma, pos):
        """EPlace::Impl::objAndGrad (src/gp/eplace.cpp:136-203) at opt-set positions pos (x then
        y) through the stage loop's own kernels: (grad, {obj, tau, hpwl, sum_wl, sum_den})."""
        pos = np.ascontiguousarray(pos, np.float32)
        grad = np.zeros_like(pos)
        out = (C.c_double * 5)()
        n = C.c_int()
        check(lib().spg_eval_grad(self.h, stage, lam, gamma, abi.fptr(pos), abi.fptr(grad), out, C.byref(n)))
        if pos.size != 2 * n.value:
            raise ValueError(f"eval_grad: {pos.size} coordinates for an opt set of {n.value} nodes")
        return grad, dict(zip(("obj", "tau", "hpwl", "sum_wl", "sum_den"), list(out)))

    # EPlace
    def run(self, stage=abi.STAGE_MGP) -> abi.Result:
        r = abi.Result()
        check(lib().spg_stage_run(self.h, stage, C.byref(r)))
        return r

    def set_iter_callback(self, fn, stride=1):
        """EPlace::setIterCallback (src/gp/eplace.h:71-72): fn(stage, iter, x, y) after the
        metrics row of every iteration with iter % stride == 0, with every node's position at
        that iteration's evaluation point (copies). fn None turns it off."""
        total = self.db.total_nodes
        if fn is None or stride <= 0:
            self._iter_cb = None
            check(lib().spg_set_iter_callback(self.h, ITER_FN(), None, 0))
            return

        def tramp(_user, stage, it, x, y):
            fn(int(stage), int(it), np.ctypeslib.as_array(x, (total,)).copy(),
               np.ctypeslib.as_array(y, (total,)).copy())

        self._iter_cb = ITER_FN(tramp)  # kept alive while registered
        check(lib().spg_set_iter_callback(self.h, self._iter_cb, None, int(stride)))

    def set_stagnation_callback(self, fn):
        """fn(stage, iter, x, y) once per mGP / cGP stage, at the iteration where the stagnation
        counter first reaches half its window (the reference's stagnation_mid diagnostic point,
        eplace.cpp:428-433), with every node's position there. None turns it off."""
        total = self.db.total_nodes
        if fn is None:
            self._mid_cb = None
            check(lib().spg_set_stagnation_callback(self.h, ITER_FN(), None))
            return

        def tramp(_user, stage, it, x, y):
            fn(int(stage), int(it), np.ctypeslib.as_array(x, (total,)).copy(),
               np.ctypeslib.as_array(y, (total,)).copy())

        self._mid_cb = ITER_FN(tramp)
        check(lib().spg_set_stagnation_callback(self.h, self._mid_cb, None))

    def eval_positions(self, which=0):
        """Every node's position at the last stage's last evaluation point (which 0) or at the
        evaluation point before it (which 1)."""
        n = self.db.total_nodes
        x, y = np.empty(n, np.float32), np.empty(n, np.float32)
        check(lib().spg_eval_positions(self.h, int(which), abi.fptr(x), abi.fptr(y)))
        return x, y

    def metrics(self, cap=100000):
        rows = (abi.IterMetrics * cap)()
        n = C.c_int()
        check(lib().spg_metrics_d2h(self.h, rows, cap, C.byref(n)))
        keys = [f[0] for f in abi.IterMetrics._fields_]
        return {k: np.array([getattr(rows[i], k) for i in range(n.value)]) for k in keys}


class EPlace:
    """EPlace (src/gp/eplace.h:56-77): construct over a PlaceDB + params, then run stages.
    The PlaceDB's positions are updated from the device after each run."""

    def __init__(self, db: PlaceDB, params: abi.Params | None = None):
        self.db = db
        self.ctx = GpContext(db, params)

    def set_iter_callback(self, fn, stride=1):
        """EPlace::setIterCallback (src/gp/eplace.h:71-72): fn(stage, iter, x, y) with every
        node's position at the evaluation point of each iteration with iter % stride == 0."""
        self._user_cb = (fn, stride) if fn is not None and stride > 0 else None
        self.ctx.set_iter_callback(fn, stride)

    def run(self, stage=abi.STAGE_MGP, metrics: list | None = None, diagnostics: str | None = None) -> abi.Result:
        """One stage from the PlaceDB's positions and flags. With a `metrics` list, the stage's
        per-iteration rows are appended to it as (stage name, rows), the input of
        superplace_b200.metrics.write_metrics_csv (the reference's MetricsSink rows). With a
        `diagnostics` directory (Config::gp_diagnostics with the sink's output directory), mGP
        and cGP write the reference's GP diagnostics there (superplace_b200.diagnostics)."""
        diag = diagnostics is not None and stage != abi.STAGE_FILLER_ONLY
        if diag:
            hooks = self._diagnostic_hooks(stage, diagnostics)
        self.ctx.set_positions(self.db.node_x, self.db.node_y)
        self.ctx.set_flags(self.db.node_flags)
        try:
            r = self.ctx.run(stage)
        finally:
            if diag:
                self.ctx.set_stagnation_callback(None)
                user = getattr(self, "_user_cb", None)
                self.ctx.set_iter_callback(*(user if user else (None, 0)))
        if metrics is not None:
            from .metrics import STAGE_NAMES

            metrics.append((STAGE_NAMES[stage], self.ctx.metrics(max(r.iterations, 1))))
        x, y = self.db.node_x, self.db.node_y
        if (x.dtype == np.float32 and y.dtype == np.float32 and x.flags.c_contiguous and y.flags.c_contiguous
                and x.flags.writeable and y.flags.writeable):
            self.ctx.positions(out=(x, y))
        else:
            x[:], y[:] = self.ctx.positions()
        if diag:
            hooks(r)
        return r

    def _diagnostic_hooks(self, stage, root):
        """Registers the first_eval and stagnation_mid points of a stage's GP diagnostics and
        returns the writer of its last_eval and delivered points (eplace.cpp:284-288,365-369,
        428-433,476-479,505-507)."""
        from . import diagnostics as D

        db, ctx, params = self.db, self.ctx, self.ctx.params
        state = {}

        def evaluation():
            if "ev" not in state:
                state["ev"] = D.Evaluation(db, params, ctx.grid_info()["dim"])
            return state["ev"]

        def point(name, it, x, y, previous, row=None, lam=None, gamma=None, step=0.0):
            if row is not None:
                rows = ctx.metrics(row + 1)
                lam, gamma, step = rows["eval_lambda"][row], rows["eval_gamma"][row], rows["step_size"][row]
            D.write_gp_diagnostic(root, stage, name, it, lam, gamma, step, db, params, ctx.grid_info()["dim"],
                                  x, y, previous, evaluation())

        def opt_positions(px, py):
            idx = D.opt_index(db, stage)
            return np.concatenate([px[idx], py[idx]])

        user = getattr(self, "_user_cb", None)

        def on_iter(st, it, x, y):
            if it == 0:
                point("first_eval", 0, x, y, None, row=0)
            if user and it % user[1] == 0:
                user[0](st, it, x, y)

        def on_mid(st, it, x, y):
            point("stagnation_mid", it, x, y, opt_positions(*ctx.eval_positions(1)), row=it)

        ctx.set_iter_callback(on_iter, user[1] if user else 1 << 30)
        ctx.set_stagnation_callback(on_mid)

        def after(r):
            try:
                delivered = (db.node_x.copy(), db.node_y.copy())
                if r.iterations > 0:
                    last = r.iterations - 1
                    lx, ly = ctx.eval_positions(0)
                    point("last_eval", last, lx, ly, opt_positions(*ctx.eval_positions(1)), row=last)
                    it = r.rollback_iter if r.stagnated else last
                    rows = ctx.metrics(last + 1)
                    point("delivered", it, delivered[0], delivered[1], opt_positions(lx, ly),
                          lam=rows["eval_lambda"][it], gamma=rows["eval_gamma"][it])
                elif r.converged:  # converged before any step (eplace.cpp:284-288)
                    g = ctx.grid_info()
                    point("delivered", -1, delivered[0], delivered[1], opt_positions(*delivered),
                          lam=r.initial_lambda, gamma=D.compute_gamma(r.initial_overflow, g["step_x"]))
            finally:
                if "ev" in state:
                    state["ev"].close()

        return after
