"""Operator parity of the CUDA path against the oracle, through the C ABI (GPU only).

Bars: integer work bit-exact (fixed-point density maps, bin indices via the maps);
gather bit-exact for cells given the same field; FP32 Poisson within 1e-5 of the FP64
oracle as max|d|/max|ref| (test/test_poisson_parity.cpp:22,54-61); WA gradient within
1e-5 of max|grad|; HPWL within 1e-12 relative; tau within 1e-6 relative.
"""
import numpy as np
import pytest

from oracle import oracle as orc
from superplace_b200 import abi, engine, generator

from . import checks
from .conftest import golden_small_db

pytestmark = pytest.mark.gpu

PARITY_TOL = 1e-5


def rel_err(ref, got):
    ref = np.asarray(ref, np.float64)
    got = np.asarray(got, np.float64)
    return np.abs(ref - got).max() / max(np.abs(ref).max(), 1e-300)


def gaussians(nx, ny):
    """Three Gaussian peaks on a 0.2 floor (test/test_poisson_parity.cpp:39-52)."""
    fx = (np.arange(nx, dtype=np.float32) + 0.5) / nx
    fy = (np.arange(ny, dtype=np.float32) + 0.5) / ny
    X, Y = np.meshgrid(fx, fy, indexing="ij")
    v = np.full((nx, ny), 0.2, np.float32)
    for cx, cy, s, a in ((0.3, 0.6, 0.05, 1.0), (0.7, 0.2, 0.12, 0.6), (0.55, 0.85, 0.02, 2.0)):
        v += a * np.exp(-((X - cx) ** 2 + (Y - cy) ** 2) / (2 * s * s))
    return v.astype(np.float32)


PARITY_GRIDS = [(64, 64, 2.5, 2.5), (512, 512, 20.88, 20.86), (1024, 1024, 10.44, 10.43),
                (256, 512, 3.0, 1.7), (512, 256, 1.7, 3.0)]


@pytest.mark.parametrize("nx,ny,sx,sy", PARITY_GRIDS)
def test_poisson_fp32_parity(nx, ny, sx, sy):
    be = engine.PoissonBackend(nx, ny, sx, sy, abi.POISSON_FP32)
    rng = np.random.default_rng(20261105 + nx * 7919 + ny)
    for rho in (rng.random((nx, ny)).astype(np.float32), gaussians(nx, ny)):
        got = be.solve(rho)
        want = orc.poisson_f64(rho, sx, sy)
        for g, w in zip(got, want):
            assert rel_err(w, g) < PARITY_TOL
        again = be.solve(rho.copy())
        for g, h in zip(got, again):
            assert np.array_equal(g, h)  # bitwise repeatable


FP64_TOL = 1e-6  # outputs are rounded once to float: ~6e-8 of max|ref|


@pytest.mark.parametrize("nx,ny,sx,sy", [(64, 64, 2.5, 2.5), (512, 512, 20.88, 20.86), (96, 160, 3.0, 1.7)])
def test_poisson_fp64_parity(nx, ny, sx, sy):
    """The FP64 form (the precision study's reference) agrees with the FP64 oracle to the
    rounding of its float outputs, on tile and non-tile grids."""
    be = engine.PoissonBackend(nx, ny, sx, sy, abi.POISSON_FP64)
    rng = np.random.default_rng(7 + nx * 31 + ny)
    for rho in (rng.random((nx, ny)).astype(np.float32), gaussians(nx, ny)):
        got = be.solve(rho)
        want = orc.poisson_f64(rho, sx, sy)
        for g, w in zip(got, want):
            assert rel_err(w, g) < FP64_TOL


def test_poisson_fp32_analytic():
    be = {}

    def solve(rho, st):
        n = rho.shape[0]
        if n not in be:
            be[n] = engine.PoissonBackend(n, n, st, st, abi.POISSON_FP32)
        return be[n].solve(rho)

    checks.poisson_analytic(solve)


def test_poisson_rejects_bad_arguments():
    with pytest.raises(engine.SpgError) as e:
        engine.PoissonBackend(1, 64, 1.0, 1.0)
    assert e.value.code == abi.SPG_E_INVALID
    with pytest.raises(engine.SpgError):
        engine.PoissonBackend(64, 64, 0.0, 1.0)


class GpuGrid:
    """BinGrid semantics through the C ABI for tests/checks.density_semantics."""

    def __init__(self, db, target, dim):
        self.ctx = engine.GpContext(db, abi.default_params(target_density=target))
        self.ctx.grid_init(target, dim)

    def accumulate(self):
        self.ctx.accumulate()
        self.tau = self.ctx.overflow()
        return (self.ctx.read_map(engine.MAP_NODE).ravel(), self.ctx.read_map(engine.MAP_FILLER).ravel())

    def overflow(self):
        return self.tau

    def total_charge(self):
        return self.ctx.total_charge()


def test_density_semantics_gpu():
    checks.density_semantics(GpuGrid)


def _check_density_bit_exact(db, dims):
    ctx = engine.GpContext(db)
    for dim in dims:
        info = ctx.grid_init(1.0, dim)
        og = orc.OracleGrid(db, 1.0, dim)
        assert info["dim"] == og.dim
        assert np.array_equal(ctx.read_map(engine.MAP_TERMINAL).ravel(), og.terminal)
        assert np.array_equal(ctx.read_map(engine.MAP_BASE).ravel(), og.base)
        ctx.accumulate()
        nf, ff, s = ctx.read_fixed()
        onf, off, os_ = og.accumulate_fixed()
        assert s == os_
        assert np.array_equal(nf, onf) and np.array_equal(ff, off)
        tau = ctx.overflow()
        otau = og.overflow(orc.fixed_to_float(onf, s))
        assert abs(tau - otau) <= 1e-6 * max(abs(otau), 1e-12)
        # repeatable bit for bit
        ctx.accumulate()
        nf2, ff2, _ = ctx.read_fixed()
        assert np.array_equal(nf, nf2) and np.array_equal(ff, ff2)


def test_density_fixed_point_bit_exact_small(small):
    db, _ = small
    _check_density_bit_exact(db, (64, 32, 128))


def test_density_fixed_point_bit_exact_large():
    db = generator.large_design(seed=3, n_cells=60_000, n_nets=63_000)
    info = engine.initialize_fillers(db, 1.0, 3)
    assert info.count > 0
    _check_density_bit_exact(db, (256,))


def test_gather_bit_exact_given_field(small):
    db, g = small
    ctx = engine.GpContext(db)
    for dim in (64, 32):
        ctx.grid_init(1.0, dim)
        ctx.write_map(engine.MAP_XI_X, g[f"d{dim}_xi_x"])
        ctx.write_map(engine.MAP_XI_Y, g[f"d{dim}_xi_y"])
        f = ctx.gather_force()
        assert np.array_equal(f, g[f"d{dim}_force"])


def test_field_after_solve_matches_oracle(small):
    db, _ = small
    ctx = engine.GpContext(db)
    info = ctx.grid_init(1.0, 64)
    ctx.accumulate()
    ctx.overflow()
    ctx.solve_field()
    rho = ctx.read_map(engine.MAP_RHO)
    og = orc.OracleGrid(db, 1.0, 64)
    nf, ff, s = og.accumulate_fixed()
    orho = og.rho(orc.fixed_to_float(nf, s), orc.fixed_to_float(ff, s)).reshape(64, 64)
    assert np.array_equal(rho, orho)
    want = orc.poisson_f64(orho, info["step_x"], info["step_y"])
    for which, w in zip((engine.MAP_PHI, engine.MAP_XI_X, engine.MAP_XI_Y), want):
        assert rel_err(w, ctx.read_map(which)) < PARITY_TOL


def test_wirelength_and_hpwl_parity(small):
    db, g = small
    ctx = engine.GpContext(db)
    for gamma in (50.0, 5.0):
        wl, grad = ctx.wa(gamma, 100)
        owl, ograd = orc.wa(db, gamma, 100)
        assert abs(wl - owl) <= 1e-6 * abs(owl)
        assert rel_err(ograd, grad) < PARITY_TOL
    assert abs(ctx.hpwl() - orc.hpwl(db)) <= 1e-12 * orc.hpwl(db)


def test_wirelength_central_differences_gpu():
    def wa(db, gamma):
        ctx = engine.GpContext(db)
        return ctx.wa(gamma, 1000)

    checks.wa_central_diff(wa)


def test_total_charge_gpu(small):
    db, g = small
    ctx = engine.GpContext(db)
    ctx.grid_init(1.0, 64)
    ctx.accumulate()
    assert abs(ctx.total_charge() - float(g["d64_charge"])) < 1e-6


def bin_index_operands(step, dim, rng):
    """Operands of int(a / step): every float within 64 ulps of each bin boundary k * step
    (k = 0..dim, the products rounded both ways), and random values over the grid and beyond."""
    s = np.float32(step)
    k = np.arange(dim + 1, dtype=np.float64)
    centres = np.concatenate([(k * float(s)).astype(np.float32), np.float32(k) * s,
                              np.nextafter((k * float(s)).astype(np.float32), np.float32(np.inf))])
    offs = np.arange(-64, 65, dtype=np.int64)
    bits = centres.view(np.int32).astype(np.int64)[:, None] + offs[None, :]
    near = bits[(bits >= 0) & (bits < 0x7F800000)].astype(np.int32).view(np.float32)
    rand = (rng.random(200_000) * (dim + 2) * float(s)).astype(np.float32)
    tiny = rng.random(1000).astype(np.float32) * np.float32(1e-30)
    return np.concatenate([near, rand, -rand[:1000], tiny, np.float32([0.0, -0.0])])


@pytest.mark.parametrize("step", [22.65625, 20.88, 0.1, 1.0 / 3.0, 3.0, 7.3e-3, 1234.567, 11600.0 / 512])
def test_bin_index_equals_float_division(step):
    """The density kernels form int(a / step) (bin_grid.cpp:49-52) as the double product
    a * (1/step) rounded to float: the same index as the float division for every operand,
    checked on the device at every bin boundary's neighbourhood and on random operands."""
    import ctypes as C

    L = engine.lib()
    L.spg_bin_index_check.argtypes = [C.c_float, C.c_void_p, C.c_int32, C.c_void_p, C.c_void_p]
    a = bin_index_operands(step, 2048, np.random.default_rng(7))
    qd = np.zeros(a.size, np.int32)
    qm = np.zeros(a.size, np.int32)
    engine.check(L.spg_bin_index_check(np.float32(step), a.ctypes.data, a.size, qd.ctypes.data, qm.ctypes.data))
    bad = np.nonzero(qd != qm)[0]
    assert bad.size == 0, (a[bad[:5]], qd[bad[:5]], qm[bad[:5]])
    # and the float division itself, as numpy forms it on the host
    host = np.trunc(a / np.float32(step)).astype(np.int64)
    ok = np.abs(host) < 2**31
    assert np.array_equal(host[ok], qd[ok])
