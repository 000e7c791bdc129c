"""The split-BF16 tensor-core (tcgen05) Poisson path against the FP64 oracle (GPU only).

Split-BF16 keeps ~16 significand bits per operand and drops the lo*lo product, so its
bar is stated separately from the FP32 path's 1e-5: max|d|/max|ref| < 3e-5 on the
reference's parity inputs (a CPU emulation of the same algorithm with exact products
predicts ~1.0e-5 max / 6e-6 RMS on the 512^2 white-noise case).
"""
import numpy as np
import pytest

from oracle import oracle as orc
from superplace_b200 import abi, engine

from . import checks
from .test_gpu_parity import gaussians, rel_err

pytestmark = pytest.mark.gpu

BF16X3_TOL = 3e-5
# the split-BF16 error grows with the contraction length (every output sums n terms, each with
# the dropped lo*lo term and the planes' rounding): at 2048 the bar is 5e-5 of max|ref|
BF16X3_TOL_2048 = 5e-5
TC_GRIDS = [(128, 128, 2.5, 2.5), (512, 512, 20.88, 20.86), (1024, 1024, 10.44, 10.43),
            (256, 512, 3.0, 1.7), (512, 256, 1.7, 3.0), (2048, 2048, 5.22, 5.21)]


@pytest.mark.parametrize("nx,ny,sx,sy", TC_GRIDS)
def test_poisson_bf16x3_parity(nx, ny, sx, sy):
    be = engine.PoissonBackend(nx, ny, sx, sy, abi.POISSON_BF16X3)
    assert be.name() == "cuda-sm100a-bf16x3"
    rng = np.random.default_rng(20261105 + nx * 7919 + ny)
    for rho in (rng.random((nx, ny)).astype(np.float32), gaussians(nx, ny)):
        got = be.solve(rho)
        want = orc.poisson_f64(rho, sx, sy)
        errs = [rel_err(w, g) for g, w in zip(got, want)]
        print(f"bf16x3 {nx}x{ny}: phi {errs[0]:.2e} xi_x {errs[1]:.2e} xi_y {errs[2]:.2e}")
        assert max(errs) < (BF16X3_TOL_2048 if max(nx, ny) >= 2048 else BF16X3_TOL)
        again = be.solve(rho.copy())
        for g, h in zip(got, again):
            assert np.array_equal(g, h)


def test_poisson_bf16x3_analytic():
    cache = {}

    def solve(rho, st):
        n = rho.shape[0]
        if n not in cache:
            cache[n] = engine.PoissonBackend(n, n, st, st, abi.POISSON_BF16X3)
        return cache[n].solve(rho)

    checks.poisson_analytic(solve, n=128)


def test_poisson_bf16x3_batched_matches_single():
    import torch

    n, b = 256, 3
    be = engine.PoissonBackend(n, n, 3.0, 3.0, abi.POISSON_BF16X3, batch=b)
    rng = np.random.default_rng(3)
    rho = rng.random((b, n, n), dtype=np.float32)
    d_rho = torch.from_numpy(rho).cuda()
    outs = [torch.empty_like(d_rho) for _ in range(3)]
    s = torch.cuda.current_stream().cuda_stream
    be.solve_device(d_rho.data_ptr(), *(o.data_ptr() for o in outs), stream=s, batch=b)
    torch.cuda.synchronize()
    for i in range(b):
        single = be.solve(rho[i])
        for o, sgl in zip(outs, single):
            assert np.array_equal(o[i].cpu().numpy(), sgl)


def test_poisson_bf16x3_wide_batched_matches_single():
    """2048 x 2048 grids run every contraction as 128 x 128 tiles (a full wave per grid): the
    choice follows one grid's problem, so a batch of two gives each grid the bits it gets
    alone."""
    import torch

    n, b = 2048, 2
    be = engine.PoissonBackend(n, n, 5.2, 5.2, abi.POISSON_BF16X3, batch=b)
    rng = np.random.default_rng(5)
    rho = rng.random((b, n, n), dtype=np.float32)
    d_rho = torch.from_numpy(rho).cuda()
    outs = [torch.empty_like(d_rho) for _ in range(3)]
    s = torch.cuda.current_stream().cuda_stream
    be.solve_device(d_rho.data_ptr(), *(o.data_ptr() for o in outs), stream=s, batch=b)
    torch.cuda.synchronize()
    for i in range(b):
        single = be.solve(rho[i])
        for o, sgl in zip(outs, single):
            assert np.array_equal(o[i].cpu().numpy(), sgl)


def test_poisson_bf16x3_rejects_untiled_grid():
    with pytest.raises(engine.SpgError) as e:
        engine.PoissonBackend(64, 64, 1.0, 1.0, abi.POISSON_BF16X3)
    assert e.value.code == abi.SPG_E_INVALID


@pytest.mark.parametrize("nx,ny", [(128, 128), (256, 256), (512, 512), (1024, 1024)])
def test_fused_solve_matches_separate_launches(nx, ny, monkeypatch):
    """A one-grid solve runs as one persistent launch (G1, the split of its output, G2, G3, G4
    with grid barriers between them) where the device holds its clusters at once; it computes
    the same tiles with the same split-K factors and reduction orders as the separate launches,
    so the results are the same bits. SPG_POISSON_FUSED=0 selects the separate launches. (Grids
    whose contractions split K over more than four CTAs, such as 256 x 512, keep the separate
    launches.)"""
    monkeypatch.setenv("SPG_POISSON_FUSED", "1")
    rng = np.random.default_rng(nx * 31 + ny)
    rho = rng.random((nx, ny)).astype(np.float32)
    be = engine.PoissonBackend(nx, ny, 1.3, 2.1, abi.POISSON_BF16X3, single_launch=True)
    n0 = engine.launch_count()
    fused = be.solve(rho)
    n_fused = engine.launch_count() - n0
    monkeypatch.setenv("SPG_POISSON_FUSED", "0")
    n0 = engine.launch_count()
    sep = be.solve(rho)
    n_sep = engine.launch_count() - n0
    assert n_sep - n_fused == 4, (n_fused, n_sep)  # G1, split, G2, G3, G4 in one launch or five
    for f, s in zip(fused, sep):
        assert np.array_equal(f, s)
    monkeypatch.setenv("SPG_POISSON_FUSED", "1")
    again = be.solve(rho)  # the barrier counters were left zeroed for the next launch
    for f, a in zip(fused, again):
        assert np.array_equal(f, a)
