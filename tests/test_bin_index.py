"""The division-free bin index on the host (CPU).

The footprint's bin indices int((lx - origin) / step) (src/gp/bin_grid.cpp:49-52) divide two
floats. The device forms the quotient as the double product a * (1/step) (1/step rounded once to
double) rounded once to float (`bin_index`, csrc/common.cuh), and relies on that being the float
quotient bit for bit: the double product is within about 2^-52 (relative) of a/step, and the
exact quotient of two floats is either a float or far enough from every midpoint between
consecutive floats that both round the same way. The GPU test checks the kernel's own
arithmetic; this one checks the claim itself with IEEE float and double arithmetic (numpy):
random operands over the magnitudes a placement grid meets, every bin boundary's float
neighbourhood, and quotients that are exactly representable.
"""
import numpy as np
import pytest


def quotient_div(a, step):
    return (a.astype(np.float32) / np.float32(step)).astype(np.float32)


def quotient_mul(a, step):
    inv = np.float64(1.0) / np.float64(np.float32(step))
    return (a.astype(np.float32).astype(np.float64) * inv).astype(np.float32)


def check(a, step):
    qd, qm = quotient_div(a, step), quotient_mul(a, step)
    bad = qd.view(np.uint32) != qm.view(np.uint32)
    assert not bad.any(), (step, a[bad][:5], qd[bad][:5], qm[bad][:5])
    # and the truncations the footprint takes
    assert np.array_equal(qd.astype(np.int64), qm.astype(np.int64))


@pytest.mark.parametrize("seed", range(4))
def test_random_operands(seed):
    rng = np.random.default_rng(seed)
    for _ in range(8):
        step = np.float32(np.exp(rng.uniform(np.log(1e-3), np.log(1e4))))
        a = (rng.uniform(-2.0, 1100.0, 1_000_000) * np.float64(step)).astype(np.float32)
        check(a, step)


@pytest.mark.parametrize("step", [22.65625, 20.859375, 11.328125, 5.2109375, 3.0, 1.7, 0.1, 12.0 / 7.0,
                                  11600.0 / 512.0, 11600.0 / 1024.0])
def test_bin_boundaries(step):
    step = np.float32(step)
    k = np.arange(0, 1025, dtype=np.float64)
    b = (k * np.float64(step)).astype(np.float32)  # the float nearest each boundary
    near = [b]
    up, down = b.copy(), b.copy()
    for _ in range(64):  # 64 floats on either side of every boundary
        up = np.nextafter(up, np.float32(np.inf))
        down = np.nextafter(down, np.float32(-np.inf))
        near += [up.copy(), down.copy()]
    check(np.concatenate(near), step)


def test_exact_quotients():
    rng = np.random.default_rng(7)
    for _ in range(16):
        step = np.float32(rng.uniform(0.01, 100.0))
        q = rng.integers(-4, 1 << 20, 200_000).astype(np.float32)
        a = (q.astype(np.float64) * np.float64(step)).astype(np.float32)
        exact = a.astype(np.float64) / np.float64(step) == np.round(a.astype(np.float64) / np.float64(step))
        check(a[exact], step)
