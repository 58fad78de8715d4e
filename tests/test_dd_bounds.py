"""Error bounds of the double-word routines the certified double-double tiers charge.

The certified double-double rungs (perm, haf / lhaf, tor) add, per operation, the
error bound of the double-word routine that produced a value:
  * accurate double-word sum (dd_add):           3u^2 / (1 - 4u) |a + b|
  * double-word plus double (dd_add_d):          2u^2 |a + b|
  * double-word product (dd_mul, FMA-based):     5u^2 |a b|
  * complex double-word product (ddc_mul):       21u^2 |x| |y|
  * division by an integer j (dd_div_d), certified a posteriori from the computed
    residual r^ = x - (q j)^:  |x - q j| <= |r^| + 4u^2 (|(q j)^| + |r^|)
(u = 2^-53; Joldes, Muller and Popescu, ACM TOMS 2017, for the first two; the
product bounds are this repository's expansion for its own FMA ordering).  This
test compiles the routines of gbskernels_b200/csrc/gbs_common.cuh (the very
__host__ __device__ source the kernels inline, through tests/dd_host.cu) for the
host and checks their errors in exact rational arithmetic on random, cancelling
and near-power-of-two operands (worst observed: 1.4, 1.2, 2.5 and 2.7 u^2).  It
needs nvcc (present wherever the library is built) but no GPU.
"""

from __future__ import annotations

import ctypes
import shutil
import subprocess
from fractions import Fraction
from pathlib import Path

import numpy as np
import pytest

HERE = Path(__file__).resolve().parent
U = Fraction(1, 2 ** 53)
N = 4000


@pytest.fixture(scope="module")
def ddlib():
    nvcc = shutil.which("nvcc") or ("/usr/local/cuda/bin/nvcc" if Path("/usr/local/cuda/bin/nvcc").exists() else None)
    if nvcc is None:
        pytest.skip("nvcc not available")
    out = HERE / "_build" / "libddhost.so"
    out.parent.mkdir(exist_ok=True)
    src = HERE / "dd_host.cu"
    hdr = HERE.parent / "gbskernels_b200" / "csrc" / "gbs_common.cuh"
    if not out.exists() or out.stat().st_mtime < max(src.stat().st_mtime, hdr.stat().st_mtime):
        cmd = [nvcc, "-x", "cu", "-O2", "-std=c++17", "-shared", "-Xcompiler", "-fPIC",
               "-Xcompiler", "-ffp-contract=off", "-gencode", "arch=compute_100a,code=sm_100a",
               "-I", str(hdr.parent), str(src), "-o", str(out)]
        subprocess.run(cmd, check=True, capture_output=True)
    lib = ctypes.CDLL(str(out))
    dp = ctypes.POINTER(ctypes.c_double)
    for name in ("t_dd_add", "t_dd_add_d", "t_dd_mul", "t_ddc_mul", "t_dd_div_resid"):
        getattr(lib, name).argtypes = [ctypes.c_int, dp, dp, dp]
        getattr(lib, name).restype = None
    return lib


def _p(a: np.ndarray):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def _call(lib, name, a, b, width):
    out = np.empty_like(a)
    getattr(lib, name)(len(a) // width, _p(np.ascontiguousarray(a)), _p(np.ascontiguousarray(b)), _p(out))
    return out


def _dw(rng, n, emin=-30, emax=30):
    """n valid double-words (hi, lo), |lo| <= ulp(hi) / 2, as a flat array."""
    hi = rng.uniform(1.0, 2.0, n) * np.exp2(rng.integers(emin, emax, n)) * rng.choice([-1.0, 1.0], n)
    # a third of them sit just above / below a power of two (where ulp changes)
    k = n // 3
    hi[:k] = np.exp2(rng.integers(emin, emax, k)) * (1.0 + rng.choice([-1.0, 1.0], k) * 2.0 ** -52 * rng.integers(0, 4, k))
    return _renorm(hi, hi * 2.0 ** -53 * rng.uniform(-1.0, 1.0, n))


def _renorm(hi: np.ndarray, lo: np.ndarray) -> np.ndarray:
    """(hi, lo) pairs normalised by Fast2Sum (|hi| >= |lo|), flat."""
    s = hi + lo
    out = np.empty(2 * len(hi))
    out[0::2], out[1::2] = s, lo - (s - hi)
    return out


def _F(x) -> Fraction:
    return Fraction(float(x))


def _val(a, i) -> Fraction:
    return _F(a[2 * i]) + _F(a[2 * i + 1])


def _worst(ratios):
    return max(ratios) if ratios else Fraction(0)


def test_dd_add_accurate_sum_bound(ddlib):
    rng = np.random.default_rng(1)
    a = _dw(rng, N)
    b = _dw(rng, N)
    # a third cancel heavily: b = -a + a small double-word
    m = N // 3
    b[0:2 * m] = _renorm(-a[0:2 * m:2], a[0:2 * m:2] * 2.0 ** -60 * rng.uniform(-1, 1, m))
    r = _call(ddlib, "t_dd_add", a, b, 2)
    bound = 3 * U ** 2 / (1 - 4 * U)
    worst = []
    for i in range(N):
        exact = _val(a, i) + _val(b, i)
        err = abs(_val(r, i) - exact)
        if exact == 0:
            assert err == 0
            continue
        worst.append(err / abs(exact))
    assert _worst(worst) <= bound, float(_worst(worst) / U ** 2)


def test_dd_add_double_bound(ddlib):
    rng = np.random.default_rng(2)
    a = _dw(rng, N)
    b = rng.uniform(1.0, 2.0, N) * np.exp2(rng.integers(-30, 30, N)) * rng.choice([-1.0, 1.0], N)
    m = N // 3
    b[:m] = -a[0:2 * m:2] * (1.0 + 2.0 ** -52 * rng.integers(-3, 4, m))
    r = _call(ddlib, "t_dd_add_d", a, b, 2)
    worst = []
    for i in range(N):
        exact = _val(a, i) + _F(b[i])
        err = abs(_val(r, i) - exact)
        if exact == 0:
            assert err == 0
            continue
        worst.append(err / abs(exact))
    assert _worst(worst) <= 2 * U ** 2, float(_worst(worst) / U ** 2)


def test_dd_mul_bound(ddlib):
    rng = np.random.default_rng(3)
    a = _dw(rng, N)
    b = _dw(rng, N)
    r = _call(ddlib, "t_dd_mul", a, b, 2)
    worst = [abs(_val(r, i) - _val(a, i) * _val(b, i)) / abs(_val(a, i) * _val(b, i)) for i in range(N)]
    assert _worst(worst) <= 5 * U ** 2, float(_worst(worst) / U ** 2)


def test_ddc_mul_bound(ddlib):
    rng = np.random.default_rng(4)
    x = np.empty(4 * N)
    y = np.empty(4 * N)
    xr, xi, yr, yi = (_dw(rng, N) for _ in range(4))
    # a third with re and im of nearly equal products (cancellation in re or im)
    m = N // 3
    xi[0:2 * m] = _renorm(xr[0:2 * m:2] * (1 + 2.0 ** -40 * rng.uniform(-1, 1, m)), xr[1:2 * m:2])
    yi[0:2 * m] = yr[0:2 * m]
    x[0::4], x[1::4], x[2::4], x[3::4] = xr[0::2], xr[1::2], xi[0::2], xi[1::2]
    y[0::4], y[1::4], y[2::4], y[3::4] = yr[0::2], yr[1::2], yi[0::2], yi[1::2]
    r = _call(ddlib, "t_ddc_mul", x, y, 4)
    worst = []
    for i in range(N):
        ar, ai = _F(x[4 * i]) + _F(x[4 * i + 1]), _F(x[4 * i + 2]) + _F(x[4 * i + 3])
        br, bi = _F(y[4 * i]) + _F(y[4 * i + 1]), _F(y[4 * i + 2]) + _F(y[4 * i + 3])
        er, ei = ar * br - ai * bi, ar * bi + ai * br
        cr, ci = _F(r[4 * i]) + _F(r[4 * i + 1]), _F(r[4 * i + 2]) + _F(r[4 * i + 3])
        # |x||y| squared, compared squared to stay rational
        mod2 = (ar * ar + ai * ai) * (br * br + bi * bi)
        err2 = (cr - er) ** 2 + (ci - ei) ** 2
        worst.append(err2 / mod2)
    assert _worst(worst) <= (21 * U ** 2) ** 2, float(_worst(worst) ** 0.5 / U ** 2)


def test_division_residual_bound(ddlib):
    rng = np.random.default_rng(5)
    x = _dw(rng, N)
    j = rng.integers(1, 33, N).astype(np.float64)
    out = np.empty(6 * N)
    ddlib.t_dd_div_resid(N, _p(x), _p(j), _p(out))
    worst = []
    for i in range(N):
        q = _F(out[6 * i]) + _F(out[6 * i + 1])
        qj = _F(out[6 * i + 2]) + _F(out[6 * i + 3])
        r = _F(out[6 * i + 4]) + _F(out[6 * i + 5])
        err = abs(_val(x, i) - q * _F(j[i]))
        slack = abs(r) + 4 * U ** 2 * (abs(qj) + abs(r))
        assert err <= slack, i
        if abs(qj):
            worst.append(abs(err - abs(r)) / abs(qj))
    # the part of the true residual the computed one misses, in units of u^2 |q j|
    assert _worst(worst) <= 4 * U ** 2, float(_worst(worst) / U ** 2)
