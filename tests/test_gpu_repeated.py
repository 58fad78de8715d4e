"""Repeated-row loop hafnian by the GPU finite-difference sieve: the reference's
golden fixtures (mpmath of the expansion), the binary128 oracle sieve, the identity
with the power-trace loop hafnian of the expanded matrix (a different algorithm and
kernel), the ordinary-hafnian case gamma = None, edge cases and the caps.
Reference test model: tests/test_repeated.py (sieve vs expansion, caps)."""

from __future__ import annotations

from pathlib import Path

import numpy as np
import pytest

from conftest import rel_err

pytestmark = pytest.mark.gpu
RNG = np.random.default_rng(99)
GOLD = Path(__file__).resolve().parent / "golden" / "golden_repeated.npz"


def base(M, scale=0.5):
    X = RNG.standard_normal((M, M)) + 1j * RNG.standard_normal((M, M))
    return scale * (X + X.T) / 2, scale * (RNG.standard_normal(M) + 1j * RNG.standard_normal(M))


def expand(A, g, r):
    idx = np.repeat(np.arange(len(r)), r)
    E = A[np.ix_(idx, idx)].copy()
    np.fill_diagonal(E, g[idx])
    return E


def test_golden_fixtures(gpu):
    rep = dict(np.load(GOLD))
    for i in range(len(rep["M"])):
        M = int(rep["M"][i])
        mp = rep["mp"][i]
        truth = complex(mp[0] + mp[1], mp[2] + mp[3])
        v = gpu.lhaf_repeated(rep["A"][i][:M, :M], rep["gamma"][i][:M], rep["reps"][i][:M])
        assert abs(v - truth) <= 1e-10 * max(abs(truth), 1e-3), (i, v, truth)


@pytest.mark.parametrize("M,maxr", [(3, 6), (4, 4), (6, 3), (8, 2)])
def test_vs_binary128_oracle_sieve(gpu, orc, M, maxr):
    A, g = base(M)
    reps = RNG.integers(0, maxr + 1, (3, M))
    reps[0, 0] = maxr  # at least one photon
    got = gpu.lhaf_repeated(A, g, reps)
    for b in range(3):
        truth = orc.lhaf_repeated(A, g, reps[b], "quad")
        assert rel_err(got[b], truth) < 1e-10 or abs(got[b] - truth) < 1e-12, (M, b, got[b], truth)


@pytest.mark.parametrize("M,maxr", [(16, 2), (32, 1)])
def test_large_patterns_vs_expanded_dd(gpu, M, maxr):
    # up to 2^32 sieve terms per pattern (many work items per pattern); the expanded
    # matrix (N <= 32) goes through the double-double power trace
    A, g = base(M, scale=0.3)
    reps = RNG.integers(0, maxr + 1, (2, M))
    reps[:, :2] = maxr
    while reps[0].sum() > 32:
        reps[0, RNG.integers(0, M)] = 0
    reps[1] = np.minimum(reps[1], 1)
    got = gpu.lhaf_repeated(A, g, reps)
    for b in range(2):
        want = gpu.lhaf(expand(A, g, reps[b]), precision="dd")
        assert rel_err(got[b], want) < 1e-10, (M, b, got[b], want)


@pytest.mark.parametrize("gamma", [True, False])
def test_equals_power_trace_of_the_expansion(gpu, gamma):
    A, g = base(10)
    if not gamma:
        g = None
    reps = np.array([[3, 0, 2, 1, 4, 0, 2, 2, 1, 3], [1, 1, 1, 1, 1, 1, 1, 1, 1, 1], [6, 6, 0, 0, 0, 0, 0, 0, 4, 0]])
    got = gpu.lhaf_repeated(A, g, reps)
    gg = np.zeros(10, np.complex128) if g is None else g
    for b in range(3):
        E = expand(A, gg, reps[b])
        want = gpu.lhaf(E, precision="dd") if g is not None else gpu.haf(E, precision="dd")
        assert rel_err(got[b], want) < 1e-10, (b, got[b], want)


def test_edge_cases_and_caps(gpu):
    A, g = base(5)
    assert gpu.lhaf_repeated(A, g, np.zeros(5, np.int32)) == 1.0
    assert gpu.lhaf_repeated(A, g, [0, 0, 1, 0, 0]) == pytest.approx(g[2], rel=1e-15)
    assert gpu.lhaf_repeated(A, None, [0, 0, 1, 0, 0]) == 0.0
    # one mode repeated twice: A_ii + gamma_i^2
    assert gpu.lhaf_repeated(A, g, [0, 2, 0, 0, 0]) == pytest.approx(A[1, 1] + g[1] ** 2, rel=1e-13)
    out = gpu.lhaf_repeated(A, g, np.zeros((0, 5), np.int32))
    assert out.shape == (0,)
    with pytest.raises(ValueError):
        gpu.lhaf_repeated(A, g, [0, -1, 0, 0, 0])
    with pytest.raises(ValueError):
        gpu.lhaf_repeated(A, g, [30, 30, 5, 0, 0])  # N = 65
    with pytest.raises(ValueError):
        gpu.lhaf_repeated(np.eye(33), None, np.ones(33, np.int32))
    B = A.copy()
    B[0, 1] = np.inf
    with pytest.raises(ValueError):
        gpu.lhaf_repeated(B, g, [1, 1, 0, 0, 0], certified=True)


# ---------------------------------------------------------------- certified sieve
def test_certified_golden_enclosures(gpu):
    rep = dict(np.load(GOLD))
    for i in range(len(rep["M"])):
        M = int(rep["M"][i])
        mp = rep["mp"][i]
        A, g, r = rep["A"][i][:M, :M], rep["gamma"][i][:M], rep["reps"][i][:M]
        v, d = gpu.lhaf_repeated(A, g, r, certified=True)
        err = abs(complex((v.real - mp[0]) - mp[1], (v.imag - mp[2]) - mp[3]))
        assert err <= d["abs_error_bound"], (i, err, d["abs_error_bound"])
        assert v == gpu.lhaf_repeated(A, g, r)  # bit-identical to the plain sieve


@pytest.mark.parametrize("M,maxr", [(3, 6), (4, 4), (6, 3), (8, 2), (12, 2)])
def test_certified_vs_binary128_oracle(gpu, orc, M, maxr):
    A, g = base(M)
    reps = RNG.integers(0, maxr + 1, (3, M))
    reps[0, 0] = maxr
    v, d = gpu.lhaf_repeated(A, g, reps, certified=True)
    plain = gpu.lhaf_repeated(A, g, reps)
    assert np.array_equal(v, plain)
    for b in range(3):
        truth = orc.lhaf_repeated(A, g, reps[b], "quad")
        bnd = d["abs_error_bound"][b]
        # the binary128 value is itself rounded to binary64 (<= u |truth| per part)
        assert abs(v[b] - truth) <= bnd + 2.3e-16 * abs(truth), (M, b, abs(v[b] - truth), bnd)
        # the sieve cancels heavily (sum |term| / |value| ~ 1e4..1e6): the bound is
        # that ratio times a few hundred u
        assert 0.0 < bnd <= 1e-6 * max(abs(truth), 1e-300) or bnd <= 1e-12, (M, b, bnd, abs(truth))


def test_certified_long_pattern_many_items(gpu):
    # 3^14 terms, 16k+ work items: the per-item incremental updates and the
    # item reduction carry their radii
    A, g = base(14, scale=0.3)
    reps = np.full(14, 2, np.int32)
    v, d = gpu.lhaf_repeated(A, g, reps, certified=True)
    want = gpu.lhaf(expand(A, g, reps), precision="dd")
    assert v == gpu.lhaf_repeated(A, g, reps)
    assert abs(v - want) <= d["abs_error_bound"] * (1 + 1e-6) + 1e-25
    assert d["abs_error_bound"] <= 1e-3 * abs(want)


def test_non_symmetric_base_matrix(gpu, orc):
    # x^T A x sees (A + A^T)/2: the sieve of a non-symmetric A equals the oracle's
    # (which forms x^T A x directly); the certified bound covers the symmetrisation
    M = 5
    A = 0.5 * (RNG.standard_normal((M, M)) + 1j * RNG.standard_normal((M, M)))
    g = 0.3 * (RNG.standard_normal(M) + 1j * RNG.standard_normal(M))
    reps = np.array([[2, 1, 3, 0, 2], [1, 1, 1, 1, 1]])
    got = gpu.lhaf_repeated(A, g, reps)
    v, d = gpu.lhaf_repeated(A, g, reps, certified=True)
    assert np.array_equal(v, got)
    for b in range(2):
        truth = orc.lhaf_repeated(A, g, reps[b], "quad")
        assert rel_err(got[b], truth) < 1e-12
        assert abs(v[b] - truth) <= d["abs_error_bound"][b] + 2.3e-16 * abs(truth)


def test_certified_edge_cases(gpu):
    A, g = base(5)
    v, d = gpu.lhaf_repeated(A, g, np.zeros(5, np.int32), certified=True)
    assert v == 1.0 and d["abs_error_bound"] == 0.0
    v, d = gpu.lhaf_repeated(A, g, [0, 0, 1, 0, 0], certified=True)
    assert abs(v - g[2]) <= d["abs_error_bound"] + 2.3e-16 * abs(g[2])
    v, d = gpu.lhaf_repeated(A, g, np.zeros((0, 5), np.int32), certified=True)
    assert v.shape == (0,)


def test_batch_equals_single_bitwise(gpu):
    A, g = base(7)
    reps = RNG.integers(0, 4, (6, 7))
    got = gpu.lhaf_repeated(A, g, reps)
    for b in range(6):
        assert gpu.lhaf_repeated(A, g, reps[b]) == got[b]
