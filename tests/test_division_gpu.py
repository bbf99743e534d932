"""The library's precomputed-reciprocal division (vof_device.cuh, div_rn_pre)
must equal CUDA's IEEE division bit for bit on every operand it can see."""
import ctypes as C
from pathlib import Path

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

LIB = Path(__file__).resolve().parent / "_build" / "libvof_divtest.so"


def run(x, d):
    if not LIB.exists():
        pytest.fail(f"{LIB} not built (__graft_entry__.build())")
    lib = C.CDLL(str(LIB))
    x = np.ascontiguousarray(x, dtype=np.float32)
    d = np.ascontiguousarray(d, dtype=np.float32)
    fast = np.empty_like(x)
    ieee = np.empty_like(x)
    P = C.POINTER(C.c_float)
    rc = lib.divtest_run(x.ctypes.data_as(P), d.ctypes.data_as(P), fast.ctypes.data_as(P),
                         ieee.ctypes.data_as(P), C.c_int(x.size))
    assert rc == 0
    return fast, ieee


def bits_equal(a, b):
    return np.array_equal(a.view(np.uint32), b.view(np.uint32)) or (
        np.array_equal(np.isnan(a), np.isnan(b)) and np.array_equal(a[~np.isnan(a)].view(np.uint32),
                                                                     b[~np.isnan(b)].view(np.uint32)))


def test_random_operands_all_exponents(cuda):
    rng = np.random.default_rng(0)
    n = 1 << 22
    with np.errstate(over="ignore"):  # exponents past float32's range give +-inf operands on purpose
        x = (rng.standard_normal(n) * np.exp2(rng.integers(-130, 130, n))).astype(np.float32)
        d = (rng.standard_normal(n) * np.exp2(rng.integers(-100, 100, n))).astype(np.float32)
    d[d == 0] = 1.0
    fast, ieee = run(x, d)
    bad = np.flatnonzero(fast.view(np.uint32) != ieee.view(np.uint32))
    bad = bad[~(np.isnan(fast[bad]) & np.isnan(ieee[bad]))]
    assert bad.size == 0, [(float(x[i]), float(d[i]), float(fast[i]), float(ieee[i])) for i in bad[:5]]


@pytest.mark.parametrize("d", [1.25e-10, 5e-4, 2.5e-7, 1.5625e-8, -9.6e5, -3.2e4, 525.0, 4e-6, 1.0e-10 * 1.03])
def test_constant_divisors_of_the_step(cuda, d):
    """Divisors of the step (cell volume, lengths, dt, Jacobi diagonals) against
    numerators spanning every binade, plus signed zeros and subnormals."""
    rng = np.random.default_rng(abs(hash(d)) % 2**32)
    n = 1 << 20
    x = (rng.uniform(1, 2, n) * np.exp2(rng.integers(-149, 127, n)) * rng.choice([-1, 1], n)).astype(np.float32)
    x[:8] = [0.0, -0.0, 1e-45, -1e-45, 1e-40, 2 ** -96, np.float32(2 ** -96) * np.float32(0.999), 3.4e38]
    dd = np.full(n, d, dtype=np.float32)
    fast, ieee = run(x, dd)
    assert np.array_equal(fast.view(np.uint32), ieee.view(np.uint32))


def test_tiny_numerators_and_subnormal_midpoints(cuda):
    """The tiny-numerator path (|x| < 2^-100: scaled quotient, one more
    rounding to the subnormal grid, midpoints settled by the remainder's sign)
    against the IEEE division: x = k 2^-149 and its neighbours over divisors
    that put x/d exactly on, just above and just below the midpoints of the
    subnormal grid, and random tiny numerators over the Jacobi diagonals of
    grids from 16 to 512 cells per side."""
    ks = np.arange(1, 1 << 14, dtype=np.float64)
    base = (ks * 2.0 ** -149).astype(np.float32)
    up = np.nextafter(base, np.float32(1))
    dn = np.nextafter(base, np.float32(0))
    xs = np.concatenate([base, up, dn, -base, -up])
    divs = [2.0, -2.0, 6.0, -6.0, 10.0, 0.375, 3.0 * 2 ** 20, -5.0 * 2 ** 23, 1.5, 2.0 ** -3, 7.0, 1.0 + 2 ** -23]
    x = np.tile(xs, len(divs))
    d = np.repeat(np.asarray(divs, dtype=np.float32), xs.size)
    fast, ieee = run(x, d)
    assert np.array_equal(fast.view(np.uint32), ieee.view(np.uint32))
    rng = np.random.default_rng(7)
    n = 1 << 20
    x = (rng.uniform(1, 2, n) * np.exp2(rng.integers(-149, -90, n)) * rng.choice([-1, 1], n)).astype(np.float32)
    h = (0.1 / rng.choice([16, 32, 48, 64, 100, 128, 200, 256, 320, 512], n)).astype(np.float32)
    c = np.float32(1.0) / h
    d = (-(c * c) * rng.choice([4, 5, 6], n).astype(np.float32)).astype(np.float32)
    fast, ieee = run(x, d)
    assert np.array_equal(fast.view(np.uint32), ieee.view(np.uint32))


def test_fp64_reciprocal_within_one_ulp(cuda):
    """vof::rcp64 (Newton-Raphson from rcp.approx.ftz.f64, used for the FP64
    partial derivatives of the adjoint) against CUDA's correctly rounded
    reciprocal, over the operands it sees (FP32 values widened to FP64: cell
    volume changes, limiter sums) and random FP64 values."""
    if not LIB.exists():
        pytest.fail(f"{LIB} not built (__graft_entry__.build())")
    lib = C.CDLL(str(LIB))
    rng = np.random.default_rng(1)
    n = 1 << 20
    x = np.concatenate([
        (rng.uniform(0.5, 2.0, n // 2) * np.exp2(rng.integers(-120, 120, n // 2))).astype(np.float32).astype(np.float64),
        rng.uniform(1.0, 2.0, n // 2) * np.exp2(rng.integers(-1000, 1000, n // 2)),
    ])
    x[::2] *= -1.0
    fast = np.empty_like(x)
    ieee = np.empty_like(x)
    P = C.POINTER(C.c_double)
    rc = lib.rcp64test_run(x.ctypes.data_as(P), fast.ctypes.data_as(P), ieee.ctypes.data_as(P), C.c_int(x.size))
    assert rc == 0
    ulp = np.spacing(np.abs(ieee))
    err = np.abs(fast - ieee) / ulp
    assert err.max() <= 1.0, err.max()
