"""Certified double-double hafnian and loop hafnian: every bound encloses the
binary128 oracle's value, the value equals the double-double tier's, and the
certified ladder escalates to it where the binary64 certificate is too loose
(reference: core/certified_dd.cu:216-328, gbskernels/__init__.py:410-425; test
model tests/test_certified.py)."""

from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
RNG = np.random.default_rng(97)


def sym(N, scale=0.5):
    X = RNG.standard_normal((N, N)) + 1j * RNG.standard_normal((N, N))
    return scale * (X + X.T) / 2


def _err(v, orc, func, A):
    """|v - f(A)| against the binary128 value carried as a double-word pair."""
    rh, rl, ih, il = getattr(orc, func)(A, "quad", hilo=True)
    return abs(complex((v.real - rh) - rl, (v.imag - ih) - il))


def _ddcert(gpu, func, mats):
    lib = gpu._lib.load()
    cm = np.ascontiguousarray(mats, dtype=np.complex128)
    B, N = cm.shape[0], cm.shape[1]
    out = np.empty(B, np.complex128)
    bnd = np.empty(B)
    gpu._lib.check(getattr(lib, f"gbs_{func}_dd_certified_host")(
        gpu._lib.dptr(cm.view(np.float64)), N, B, gpu._lib.dptr(out.view(np.float64)), gpu._lib.dptr(bnd)),
        f"gbs_{func}_dd_certified_host")
    return out, bnd


@pytest.mark.parametrize("func,N", [("haf", 2), ("haf", 6), ("haf", 10), ("haf", 16), ("haf", 20),
                                    ("lhaf", 3), ("lhaf", 8), ("lhaf", 13), ("lhaf", 18)])
def test_dd_certified_vs_binary128(gpu, orc, func, N):
    mats = np.stack([sym(N), sym(N, 1.5)])
    out, bnd = _ddcert(gpu, func, mats)
    dd = getattr(gpu, f"{func}_batched")(mats, precision="dd")
    for i in range(len(mats)):
        truth = getattr(orc, func)(mats[i], "quad")
        e = _err(out[i], orc, func, mats[i])
        assert np.isfinite(bnd[i]) and bnd[i] >= 0
        assert e <= bnd[i], (func, N, i, e, bnd[i])
        assert bnd[i] <= 1e-14 * abs(truth), (func, N, i, bnd[i] / abs(truth))
        assert out[i] == dd[i]  # the certified double-double value is the dd value


def test_dd_certified_multi_item(gpu, orc):
    # N = 24: 2^12 subsets over 64 work items, partials summed in double-word
    A = sym(24, 0.4)
    out, bnd = _ddcert(gpu, "haf", A[None])
    truth = orc.haf(A, "quad")
    assert _err(out[0], orc, "haf", A) <= bnd[0]
    assert bnd[0] <= 1e-14 * abs(truth)
    assert out[0] == gpu.haf_batched(A[None], precision="dd")[0]


def test_dd_certified_exact_cases(gpu, orc):
    # haf(J_{2n}) = (2n-1)!!, lhaf(J_N) = the telephone numbers, odd N haf = 0
    J = np.ones((8, 8), np.complex128)
    out, bnd = _ddcert(gpu, "haf", J[None])
    assert abs(out[0] - 105.0) <= bnd[0] and bnd[0] <= 1e-13
    J7 = np.ones((7, 7), np.complex128)
    out, bnd = _ddcert(gpu, "lhaf", J7[None])
    assert abs(out[0] - 232.0) <= bnd[0] and bnd[0] <= 1e-12
    out, bnd = _ddcert(gpu, "haf", J7[None])
    assert out[0] == 0 and bnd[0] == 0


def test_haf_certified_ladder_escalates_to_dd(gpu):
    mats = np.stack([sym(14) for _ in range(3)])
    v, d = gpu.haf_batched(mats, precision="certified", return_diagnostics=True, rtol=1e-15)
    dd = gpu.haf_batched(mats, precision="dd")
    for i in range(3):
        assert d[i]["rel_error_bound"] <= 1e-15
        if d[i]["tier"] == "certified-dd":
            assert d[i]["escalated"] is True and v[i] == dd[i]
    assert any(x["tier"] == "certified-dd" for x in d)


def test_lhaf_dd_certified_in_mixed_queue(gpu):
    # the certified double-double tier inside a mixed persistent queue equals the
    # one-shot value and bound
    mats = [sym(10), sym(9), sym(12)]
    funcs = ["lhaf", "haf", "haf"]
    with gpu.Workspace() as ws:
        r = ws.evaluate_resident(funcs, mats, ["certified-dd", "fp64", "certified-dd"])
        vals, aux = r.numpy(), r.aux.numpy()
        r.close()
    o0, b0 = _ddcert(gpu, "lhaf", mats[0][None])
    o2, b2 = _ddcert(gpu, "haf", mats[2][None])
    assert vals[0] == o0[0] and aux[0] == b0[0]
    assert vals[2] == o2[0] and aux[2] == b2[0]
