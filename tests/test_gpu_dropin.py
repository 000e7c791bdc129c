"""The drop-in, compiled: the reference's own test programs run against the reference-side
adapters of this engine (GPU only).

oracle/Makefile builds three programs from the reference's sources where they lie, each linked
with an adapter of oracle/ref_shim/ over superplace_b200/libspgpu.so:

  test_poisson_sm100a         test/test_poisson.cpp, unmodified: its six analytic checks
                              (Gaussian field, uniform density, symmetry, round trip, field =
                              -grad phi, determinism) through PoissonBackend::solve, once on the
                              CPU backend and once on the device backend the reference's own
                              factory (poisson_factory.cpp, ENABLE_CUDA) hands out;
  test_poisson_parity_sm100a  test/test_poisson_parity.cpp, unmodified: device against CPU
                              backend, max|d| / max|CPU| < 1e-5 on its five grids;
  test_eplace_sm100a          test/test_eplace.cpp, unmodified, over a device-backed sp::EPlace
                              (ref_shim/sm100a_eplace.cpp in place of src/gp/eplace.cpp): the
                              reference's mGP regression checks on the device loop.

test_poisson asserts the backends' names ("cpu-fftw" for FFTW's CPU backend, "cuda-cufft" for
its cuFFT one). Here the CPU backend is the FFT stand-in for FFTW and the device backend is this
engine's, so exactly those two name checks fail and every other check must pass.
"""
import os
import re
import subprocess

import pytest

from .conftest import ROOT

pytestmark = pytest.mark.gpu

BIN = os.path.join(ROOT, "oracle", "_ref")


def run(name, timeout=900, env=None):
    exe = os.path.join(BIN, name)
    if not os.path.exists(exe):
        pytest.skip(f"oracle/_ref/{name} not built")
    e = dict(os.environ)
    e.update(env or {})
    out = subprocess.run([exe], capture_output=True, text=True, timeout=timeout, env=e)
    return out.returncode, out.stdout, out.stderr


def failures(stderr):
    """(file:line, expr) of every FAIL report of the reference's test_util.h."""
    return re.findall(r"FAIL (\S+)\n\s+expr : (.*)", stderr)


def test_reference_poisson_checks_on_the_device_backend():
    rc, out, err = run("test_poisson_sm100a")
    fails = failures(err)
    assert "backend: cuda-sm100a" in out, out  # the second pass ran on the device backend
    assert all("name()" in expr for _, expr in fails), fails
    assert len(fails) == 2, (fails, out)


def test_reference_poisson_parity_on_the_device_backend():
    rc, out, err = run("test_poisson_parity_sm100a")
    assert rc == 0 and "[PASS] test_poisson_parity" in out, out + err


def test_reference_eplace_checks_on_the_device_engine():
    rc, out, err = run("test_eplace_sm100a")
    assert rc == 0 and "[PASS] test_eplace" in out, out + err
