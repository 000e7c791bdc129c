"""ctypes mirror of the structs declared in include/spgpu.h (the C ABI of the engine).

The layouts must match include/spgpu.h field for field; tests/test_abi.py checks the
sizes against the library's own view of them.
"""
import ctypes as C

SPG_OK = 0
SPG_E_INVALID = -1
SPG_E_NO_DEVICE = -2
SPG_E_CUDA = -3
SPG_E_NON_FINITE = -4
SPG_E_OUT_OF_CORE = -5
SPG_E_CONVERGENCE = -6
SPG_E_ROLLBACK = -7
SPG_E_STATE = -8
SPG_E_CAPACITY = -9

F_MACRO, F_FIXED, F_FILLER, F_NI = 1, 2, 4, 8

POISSON_FP32 = 0
POISSON_BF16X3 = 1
POISSON_FP64 = 2

STAGE_MGP, STAGE_FILLER_ONLY, STAGE_CGP = 0, 1, 2

# InvariantError kinds of the reference (src/util/invariant.h:10-19) by status code.
ERROR_KINDS = {
    SPG_E_NON_FINITE: "non_finite",
    SPG_E_OUT_OF_CORE: "out_of_core",
    SPG_E_CONVERGENCE: "convergence_mismatch",
    SPG_E_ROLLBACK: "rollback_mismatch",
}

_fp = C.POINTER(C.c_float)
_ip = C.POINTER(C.c_int32)
_u8p = C.POINTER(C.c_uint8)


class DbView(C.Structure):
    _fields_ = [
        ("num_movable", C.c_int32), ("num_nodes", C.c_int32), ("num_fillers", C.c_int32),
        ("node_x", _fp), ("node_y", _fp), ("node_w", _fp), ("node_h", _fp),
        ("node_flags", _u8p),
        ("num_pins", C.c_int32),
        ("pin_offset_x", _fp), ("pin_offset_y", _fp), ("pin2node", _ip), ("pin2net", _ip),
        ("num_nets", C.c_int32),
        ("net2pin_start", _ip), ("flat_net2pin", _ip), ("node2pin_start", _ip),
        ("flat_node2pin", _ip),
        ("num_rows", C.c_int32),
        ("row_ly", _fp), ("row_height", _fp), ("row_lx", _fp), ("row_step", _fp),
        ("row_num_sites", _ip),
        ("core_lx", C.c_float), ("core_ly", C.c_float), ("core_hx", C.c_float),
        ("core_hy", C.c_float), ("row_height_mode", C.c_float), ("total_row_area", C.c_double),
    ]


class Params(C.Structure):
    _fields_ = [
        ("target_density", C.c_float), ("target_overflow", C.c_float),
        ("cgp_target_overflow", C.c_float), ("gp_max_iter", C.c_int32),
        ("ignore_net_degree", C.c_int32), ("gp_bin_dim", C.c_int32),
        ("filler_only_iters", C.c_int32), ("delta_hpwl_ref", C.c_float),
        ("lambda_schedule_relative", C.c_int32), ("delta_hpwl_relative", C.c_double),
        ("use_bb", C.c_int32), ("gp_backtrack", C.c_int32), ("max_backtrack", C.c_int32),
        ("gp_stagnation_window", C.c_int32), ("gp_stagnation_min_gain", C.c_float),
        ("random_seed", C.c_uint64), ("poisson_precision", C.c_int32), ("verbose", C.c_int32),
        ("freeze_lambda", C.c_int32), ("freeze_gamma", C.c_int32), ("poisson_single_launch", C.c_int32),
    ]


class Result(C.Structure):
    _fields_ = [
        ("iterations", C.c_int32), ("hpwl", C.c_double), ("overflow", C.c_float),
        ("converged", C.c_int32), ("stagnated", C.c_int32), ("rollback_iter", C.c_int32),
        ("evaluations", C.c_int64), ("elapsed_ms", C.c_double), ("initial_hpwl", C.c_double),
        ("initial_overflow", C.c_float), ("initial_lambda", C.c_float),
    ]


class IterMetrics(C.Structure):
    _fields_ = [
        ("iter", C.c_int32), ("hpwl", C.c_double), ("overflow", C.c_float),
        ("lambda_", C.c_float), ("gamma", C.c_float), ("step_size", C.c_float),
        ("grad_norm_wl", C.c_float), ("grad_norm_den", C.c_float),
        ("eval_lambda", C.c_float), ("eval_gamma", C.c_float), ("delta_hpwl", C.c_double),
        ("lambda_mu", C.c_float), ("evaluations", C.c_int64),
        ("max_displacement", C.c_float), ("elapsed_ms", C.c_double),
    ]


class FillerInfo(C.Structure):
    _fields_ = [
        ("count", C.c_int32), ("width", C.c_float), ("height", C.c_float),
        ("whitespace_area", C.c_double), ("node_area_scaled", C.c_double),
        ("total_filler_area", C.c_double),
    ]


def default_params(**overrides) -> Params:
    """configs/default.json of the reference, as an spg_params struct."""
    p = Params(
        target_density=1.0, target_overflow=0.10, cgp_target_overflow=0.10,
        gp_max_iter=2000, ignore_net_degree=100, gp_bin_dim=0, filler_only_iters=20,
        delta_hpwl_ref=3.5e5, lambda_schedule_relative=0, delta_hpwl_relative=0.01,
        use_bb=1, gp_backtrack=1, max_backtrack=10, gp_stagnation_window=200,
        gp_stagnation_min_gain=0.02, random_seed=1002, poisson_precision=POISSON_FP32,
        verbose=0, freeze_lambda=0, freeze_gamma=0, poisson_single_launch=0,
    )
    for k, v in overrides.items():
        if not hasattr(p, k):
            raise KeyError(k)
        setattr(p, k, v)
    return p


def fptr(a):
    return a.ctypes.data_as(_fp)


def iptr(a):
    return a.ctypes.data_as(_ip)


def u8ptr(a):
    return a.ctypes.data_as(_u8p)
