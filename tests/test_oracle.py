"""Pins the oracle (oracle/sp_oracle.c) before it is trusted as the checker of the CUDA path:

* bit-level against fixtures produced by the reference's own code (tests/golden/),
* against the reference's own known-answer tests (tests/checks.py),
* against scipy's DCT for the FP64 Poisson solve,
* live against oracle/_ref when it is built (the reference compiled from its sources).
"""
import numpy as np
import pytest
import scipy.fft as sf

from oracle import oracle as orc
from oracle import ref

from . import checks
from .conftest import golden_small_db, load_golden


def test_static_density_bit_exact(small):
    db, g = small
    for dim in (64, 32):
        og = orc.OracleGrid(db, 1.0, dim)
        info = g[f"d{dim}_info"]
        assert og.dim == int(info[0])
        assert np.float32(og.g.step_x) == np.float32(info[1])
        assert og.g.movable_area_scaled == float(g[f"d{dim}_den"])
        assert np.array_equal(og.terminal, g[f"d{dim}_terminal"].ravel())
        assert np.array_equal(og.base, g[f"d{dim}_base"].ravel())


def test_accumulate_overflow_charge_bit_exact(small):
    db, g = small
    for dim in (64, 32):
        og = orc.OracleGrid(db, 1.0, dim)
        node, filler = og.accumulate_chunks(8)
        assert np.array_equal(node, g[f"d{dim}_node"].ravel())
        assert np.array_equal(filler, g[f"d{dim}_filler"].ravel())
        assert og.overflow(node) == float(g[f"d{dim}_tau"])
        assert og.total_charge() == float(g[f"d{dim}_charge"])


def test_fixed_point_accumulate_conserves_charge(small):
    db, g = small
    og = orc.OracleGrid(db, 1.0, 64)
    nf, ff, s = og.accumulate_fixed()
    assert 30 <= s <= 40
    node = g["d64_node"].ravel().astype(np.float64)
    fixed = orc.fixed_to_float(nf, s).astype(np.float64)
    assert np.abs(fixed - node).max() <= 1e-6 * node.max()
    # exact integer sum of rounded contributions vs the reference's double total charge
    total = (nf.sum() + ff.sum()) * np.ldexp(1.0, -s)
    assert abs(total - float(g["d64_charge"])) < 1e-6


def test_gather_bit_exact(small):
    db, g = small
    for dim in (64, 32):
        og = orc.OracleGrid(db, 1.0, dim)
        f = og.gather(g[f"d{dim}_xi_x"], g[f"d{dim}_xi_y"])
        assert np.array_equal(f, g[f"d{dim}_force"])


def test_wirelength_hpwl_gamma_bit_exact(small):
    db, g = small
    for gamma in (50.0, 5.0):
        wl, grad = orc.wa(db, gamma, 100)
        assert wl == float(g[f"wa{int(gamma)}_wl"])
        assert np.array_equal(grad, g[f"wa{int(gamma)}_grad"])
    assert orc.hpwl(db) == float(g["hpwl"])
    for t, v in zip(g["gamma_tau"], g["gamma_val"]):
        assert orc.gamma(float(t), 9.375) == v


def test_oracle_density_semantics():
    class G:
        def __init__(self, db, target, dim):
            self.og = orc.OracleGrid(db, target, dim)
            self.node = None

        def accumulate(self):
            nf, ff, s = self.og.accumulate_fixed()
            self.node = orc.fixed_to_float(nf, s)
            return self.node, orc.fixed_to_float(ff, s)

        def overflow(self):
            return self.og.overflow(self.node)

        def total_charge(self):
            return self.og.total_charge()

    checks.density_semantics(G)


def test_oracle_poisson_analytic():
    checks.poisson_analytic(lambda rho, st: tuple(a.astype(np.float32) for a in orc.poisson_f64(rho, st, st)))


def test_oracle_poisson_matches_scipy():
    rng = np.random.default_rng(5)
    for nx, ny, sx, sy in ((64, 64, 2.5, 2.5), (32, 48, 3.0, 1.7), (128, 64, 1.7, 3.0)):
        rho = rng.random((nx, ny))
        phi, ex, ey = orc.poisson_f64(rho, sx, sy)
        F = sf.dct(sf.dct(rho, type=2, axis=0), type=2, axis=1)
        u = np.pi * np.arange(nx) / (nx * sx)
        v = np.pi * np.arange(ny) / (ny * sy)
        den = u[:, None] ** 2 + v[None, :] ** 2
        den[0, 0] = 1.0
        P = F / (4.0 * nx * ny) / den
        P[0, 0] = 0.0
        phi_s = sf.dct(sf.dct(P, type=3, axis=0), type=3, axis=1)
        # xi_x = 2 sum_{j>=1} u_j P_j sin(.) ; scipy dst type 3 of the shifted coefficients
        Q = np.zeros_like(P)
        Q[:-1] = P[1:] * u[1:, None]
        ex_s = sf.dct(sf.dst(Q, type=3, axis=0), type=3, axis=1)
        R = np.zeros_like(P)
        R[:, :-1] = P[:, 1:] * v[None, 1:]
        ey_s = sf.dst(sf.dct(R, type=3, axis=0), type=3, axis=1)
        for a, b in ((phi, phi_s), (ex, ex_s), (ey, ey_s)):
            assert np.abs(a - b).max() <= 1e-12 * np.abs(b).max()


def test_oracle_wirelength_central_differences():
    checks.wa_central_diff(lambda db, gamma: orc.wa(db, gamma, 1000))


@pytest.mark.skipif(not ref.available(), reason="oracle/_ref not built")
def test_oracle_matches_reference_build_live():
    """A second design (other seed) through the oracle and the reference's own code."""
    from superplace_b200 import generator

    db = generator.small_design(7)
    r = ref.RefDb(db)
    info = r.fillers_init(1.0, 7)
    x, y, _, _, _ = r.nodes()
    db.set_fillers(int(info[0]), info[1], info[2], x[db.num_nodes:], y[db.num_nodes:])
    for dim in (0, 16, 128):
        rg = ref.RefGrid(r, 1.0, dim)
        og = orc.OracleGrid(db, 1.0, dim)
        assert rg.dim == og.dim
        assert np.array_equal(rg.read(2).ravel(), og.terminal)
        assert np.array_equal(rg.read(3).ravel(), og.base)
        rg.accumulate()
        n1, f1 = og.accumulate_chunks(8)
        assert np.array_equal(rg.read(0).ravel(), n1) and np.array_equal(rg.read(1).ravel(), f1)
        assert rg.overflow() == og.overflow(n1)
        rg.solve()
        assert np.array_equal(rg.gather(), og.gather(rg.read(6), rg.read(7)))
    wl_r, g_r = r.wa(20.0)
    wl_o, g_o = orc.wa(db, 20.0)
    assert wl_r == wl_o and np.array_equal(g_r, g_o)
    assert r.hpwl() == orc.hpwl(db)


@pytest.mark.skipif(not ref.available(), reason="oracle/_ref not built")
def test_reference_shim_poisson_agrees_with_oracle():
    """The FFT stand-in used for the reference's CPU path vs the FP64 oracle, on the
    reference's parity grids (test/test_poisson_parity.cpp:122-128), at 1e-5."""
    rng = np.random.default_rng(20261105)
    for nx, ny, sx, sy in ((64, 64, 2.5, 2.5), (512, 512, 20.88, 20.86), (256, 512, 3.0, 1.7)):
        rho = rng.random((nx, ny)).astype(np.float32)
        a = ref.poisson(rho, sx, sy)
        b = orc.poisson_f64(rho, sx, sy)
        for p, q in zip(a, b):
            assert np.abs(p - q).max() / np.abs(q).max() < 1e-5


def test_nesterov_golden_shape():
    """The reference optimizer's known answers used by the device optimizer tests."""
    g = load_golden("nesterov.npz")
    assert g["huge_bt1_meta"][1] == g["huge_bt0_meta"][1] + 1  # exactly one re-evaluation
    assert g["huge_bt1_meta"][0] < 1e-6 < 1e3 < g["huge_bt0_meta"][0]
    assert np.array_equal(g["iso_bt0_pos"], g["iso_bt1_pos"])  # backtracking is a no-op


def test_golden_db_roundtrip():
    db, g = golden_small_db(False)
    assert db.num_movable == 2000 and db.num_nodes == 2064
    assert db.net2pin_start[-1] == db.num_pins
