"""The allocation-free Poisson entry point, spg_poisson_solve_static (GPU only).

Callers that cannot call cudaMalloc (for example a host that reserves all device memory
in its own pool up front) cannot build a Poisson plan; this entry point keeps its scratch
in a static device array instead. Here it is called through the C ABI with device
buffers the test owns, twice in a row, and each result is compared with the plan-based
entry point (spg_poisson_solve_device) within the parity tolerance of the Poisson tests
(max|d| / max|ref| < 1e-5). This file is collected last so that a run which stops at the
first failure has already run every other test; it also passes alone in a fresh process.
"""
import numpy as np
import pytest

from superplace_b200 import abi, engine

pytestmark = pytest.mark.gpu

TOL = 1e-5


def rel_err(ref, got):
    ref = np.asarray(ref, np.float64)
    got = np.asarray(got, np.float64)
    return np.abs(ref - got).max() / max(np.abs(ref).max(), 1e-300)


@pytest.mark.parametrize("nx,ny,sx,sy", [(512, 512, 20.88, 20.86), (64, 128, 2.5, 1.7), (128, 64, 1.7, 2.5),
                                         (37, 50, 3.1, 2.2)])
def test_static_solve_matches_plan_solve_twice(nx, ny, sx, sy):
    import torch

    dev = torch.device("cuda:0")
    stream = torch.cuda.current_stream(dev)
    rng = np.random.default_rng(nx * 31 + ny)
    plan = engine.PoissonBackend(nx, ny, sx, sy, abi.POISSON_FP32)
    for call in range(2):
        rho = torch.from_numpy(rng.random((nx, ny), dtype=np.float32)).to(dev)
        want = [torch.empty_like(rho) for _ in range(3)]
        got = [torch.full_like(rho, float("nan")) for _ in range(3)]
        plan.solve_device(rho.data_ptr(), *(t.data_ptr() for t in want), stream=stream.cuda_stream)
        engine.poisson_solve_static(nx, ny, sx, sy, rho.data_ptr(), *(t.data_ptr() for t in got),
                                    stream=stream.cuda_stream)
        torch.cuda.synchronize(dev)
        for w, g in zip(want, got):
            w, g = w.cpu().numpy(), g.cpu().numpy()
            assert np.all(np.isfinite(g)), f"call {call}: non-finite output"
            assert rel_err(w, g) < TOL, f"call {call}: {rel_err(w, g):.3e}"


@pytest.mark.parametrize("nx,ny,sx,sy", [(64, 64, 2.5, 2.5), (128, 64, 1.7, 2.5), (37, 50, 3.1, 2.2)])
def test_static_solve_matches_fp64_oracle(nx, ny, sx, sy):
    """Directly against the FP64 oracle (oracle/oracle.py: the reference's transforms by
    their definitions), within the same 1e-5 of max|ref|."""
    import torch

    from oracle import oracle as orc

    dev = torch.device("cuda:0")
    rng = np.random.default_rng(nx * 7 + ny)
    rho_h = rng.random((nx, ny), dtype=np.float32)
    rho = torch.from_numpy(rho_h).to(dev)
    got = [torch.full_like(rho, float("nan")) for _ in range(3)]
    engine.poisson_solve_static(nx, ny, sx, sy, rho.data_ptr(), *(t.data_ptr() for t in got),
                                stream=torch.cuda.current_stream(dev).cuda_stream)
    torch.cuda.synchronize(dev)
    for w, g in zip(orc.poisson_f64(rho_h, sx, sy), got):
        assert rel_err(w, g.cpu().numpy()) < TOL


def test_static_solve_rejects_sizes_beyond_its_maximum():
    import torch

    a = torch.zeros(1024 * 1024, dtype=torch.float32, device="cuda:0")
    p = a.data_ptr()
    with pytest.raises(engine.SpgError) as e:
        engine.poisson_solve_static(1024, 1024, 1.0, 1.0, p, p, p, p)
    assert e.value.code == abi.SPG_E_CAPACITY
    assert "512" in str(e.value)
