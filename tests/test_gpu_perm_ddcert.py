"""Certified double-double permanent: the ball-arithmetic form of the double-double
Glynn walk.  Every bound encloses the binary128 oracle's value, the value equals
the double-double tier's, and the certified ladder escalates to it where the
binary64 certificate is too loose (reference: core/certified_dd.cu:124-201,
gbskernels/__init__.py:410-425; test model tests/test_certified.py)."""

from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
RNG = np.random.default_rng(91)


def haar(n):
    Z = (RNG.standard_normal((n, n)) + 1j * RNG.standard_normal((n, n))) / np.sqrt(2)
    Q, R = np.linalg.qr(Z)
    return Q * (np.diag(R) / np.abs(np.diag(R)))


def _err(v, orc, A):
    """|v - perm(A)| against the binary128 value carried as a double-word pair."""
    rh, rl, ih, il = orc.perm(A, "quad", hilo=True)
    return abs(complex((v.real - rh) - rl, (v.imag - ih) - il))


def _ddcert(gpu, mats):
    lib = gpu._lib.load()
    cm = np.ascontiguousarray(mats, dtype=np.complex128)
    B, n = cm.shape[0], cm.shape[1]
    out = np.empty(B, np.complex128)
    bnd = np.empty(B)
    gpu._lib.check(lib.gbs_perm_dd_certified_host(gpu._lib.dptr(cm.view(np.float64)), n, B,
                                                  gpu._lib.dptr(out.view(np.float64)), gpu._lib.dptr(bnd)),
                   "gbs_perm_dd_certified_host")
    return out, bnd


@pytest.mark.parametrize("n", [1, 2, 5, 6, 9, 12, 16])
def test_perm_dd_certified_vs_binary128(gpu, orc, n):
    mats = np.stack([haar(n), 0.7 * (RNG.standard_normal((n, n)) + 1j * RNG.standard_normal((n, n)))])
    out, bnd = _ddcert(gpu, mats)
    dd = gpu.perm_batched(mats, precision="dd")
    for i in range(len(mats)):
        truth = orc.perm(mats[i], "quad")
        assert np.isfinite(bnd[i]) and bnd[i] >= 0
        assert _err(out[i], orc, mats[i]) <= bnd[i], (n, i, _err(out[i], orc, mats[i]), bnd[i])
        # the bound is the final rounding to binary64 plus a double-word walk
        assert bnd[i] <= 1e-14 * abs(truth), (n, i, bnd[i] / abs(truth))
        assert out[i] == dd[i]  # the certified double-double value is the dd value


def test_perm_dd_certified_multi_item(gpu, orc):
    # n = 20: 2^19 Gray steps over many work items, the partials summed in double-word
    A = haar(20)
    out, bnd = _ddcert(gpu, A[None])
    truth = orc.perm(A, "quad")
    assert _err(out[0], orc, A) <= bnd[0]
    assert bnd[0] <= 1e-14 * abs(truth)
    assert out[0] == gpu.perm_batched(A[None], precision="dd")[0]


def test_perm_dd_certified_cancellation_and_zero(gpu, orc):
    # a block matrix with a zero permanent (the block [[1, 1], [1, -1]] has
    # permanent 0) and a heavily cancelling +-1 matrix
    Z = np.array([[1, 1, 0, 0], [1, -1, 0, 0], [0, 0, 1, 1], [0, 0, 1, 1]], np.complex128)
    S = np.where(RNG.random((10, 10)) < 0.5, -1.0, 1.0).astype(np.complex128)
    for M in (Z, S):
        out, bnd = _ddcert(gpu, M[None])
        assert _err(out[0], orc, M) <= bnd[0]
        assert bnd[0] <= 1e-12 * max(1.0, np.abs(M).sum())


def test_perm_certified_ladder_escalates_to_dd(gpu):
    mats = np.stack([haar(16) for _ in range(3)])
    v, d = gpu.perm_batched(mats, precision="certified", return_diagnostics=True, rtol=1e-15)
    dd = gpu.perm_batched(mats, precision="dd")
    for i in range(3):
        assert d[i]["rel_error_bound"] <= 1e-15
        if d[i]["tier"] == "certified-dd":
            assert d[i]["escalated"] is True and v[i] == dd[i]
    assert any(x["tier"] == "certified-dd" for x in d)


def test_perm_dd_certified_rejects_non_finite(gpu):
    A = haar(4)
    A[1, 2] = np.nan
    with pytest.raises(Exception):
        _ddcert(gpu, A[None])
