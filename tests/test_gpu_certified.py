"""Certified tier: every bound encloses the ground truth (mpmath from the reference,
or the binary128 oracle) and the value is bit-identical to the fp64 tier.
Reference test model: tests/test_certified.py (enclosure on closed forms, random and
adversarial inputs; fail-closed refusals)."""

from __future__ import annotations

import numpy as np
import pytest

from conftest import golden_cases

pytestmark = pytest.mark.gpu
RNG = np.random.default_rng(77)


def sym(N, scale=0.5):
    X = RNG.standard_normal((N, N)) + 1j * RNG.standard_normal((N, N))
    return scale * (X + X.T) / 2


def phys_O(n):
    X = RNG.standard_normal((2 * n, 2 * n))
    S = X @ X.T / (2 * n) + np.eye(2 * n)
    O = np.eye(2 * n) - np.linalg.inv(S)
    return (O + O.T) / 2


def _cert(G, func, mats):
    vals, diags = getattr(G, f"{func}_batched")(mats, precision="certified", return_diagnostics=True)
    return vals, np.array([d["abs_error_bound"] for d in diags])


@pytest.mark.parametrize("func", ["perm", "haf", "lhaf", "tor"])
def test_golden_enclosures(gpu, golden, func):
    for m, truth, _, i in golden_cases(golden, func):
        if func == "tor" and np.any(np.imag(m) != 0):
            continue
        v, b = _cert(gpu, func, m[None])
        assert np.isfinite(b[0]) and b[0] >= 0
        assert abs(v[0] - truth) <= b[0], (func, i, abs(v[0] - truth), b[0])
        assert v[0] == getattr(gpu, f"{func}_batched")(m[None])[0]  # bit-identical to fp64


@pytest.mark.parametrize("func,size", [("haf", 12), ("haf", 18), ("lhaf", 11), ("lhaf", 16),
                                       ("perm", 12), ("perm", 15), ("tor", 8), ("tor", 12)])
def test_enclosures_vs_binary128(gpu, orc, func, size):
    if func == "perm":
        mats = RNG.standard_normal((3, size, size)) + 1j * RNG.standard_normal((3, size, size))
    elif func == "tor":
        mats = np.stack([phys_O(size) for _ in range(3)])
    else:
        mats = np.stack([sym(size) for _ in range(3)])
    v, b = _cert(gpu, func, mats)
    fp = getattr(gpu, f"{func}_batched")(mats)
    assert np.array_equal(v, fp)
    for i in range(3):
        truth = getattr(orc, func)(mats[i], "quad")
        err = abs(v[i] - truth)
        assert err <= b[i], (func, size, i, err, b[i])
        assert b[i] <= 1e-6 * max(abs(truth), 1e-300), (func, size, i, b[i] / abs(truth))


def test_tor_uncertifiable_fails_closed(gpu):
    O = np.stack([phys_O(3), 1.5 * np.eye(6)])
    with pytest.raises(FloatingPointError):
        gpu.tor_batched(O, precision="certified", return_diagnostics=True)
    v, d = gpu.tor(O[0], precision="certified", return_diagnostics=True)
    assert d["tier"] == "certified-fp64" and d["rel_error_bound"] < 1e-10


def test_certified_rtol_diagnostics(gpu):
    A = sym(10)
    v, d = gpu.haf(A, precision="certified", return_diagnostics=True, rtol=1e-3)
    assert d["escalated"] is False and d["rel_error_bound"] <= 1e-3
