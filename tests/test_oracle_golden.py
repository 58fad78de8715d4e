"""Pin the CPU oracle before trusting it (CPU only).

The oracle (oracle/gbs_oracle.cpp) is this repository's restatement of the
reference algorithms.  It is checked against
  * the reference's own mpmath ground truth and binary64 CPU values, committed as
    tests/golden/golden.npz by tests/golden/make_golden.py,
  * the reference's closed forms (tests/test_layer1_combinatorial.py:25-77,
    tests/test_hafnian_layer1.py:29-81, tests/test_loop_hafnian.py:28-51,
    tests/test_torontonian.py:32-48 in the reference),
  * the reference's own kernels compiled on the host (oracle/_ref, when built).
"""

from __future__ import annotations

import math

import numpy as np
import pytest

from conftest import golden_cases, rel_err


@pytest.mark.parametrize("func", ["perm", "haf", "lhaf", "tor"])
def test_oracle_fp64_matches_reference_mpmath(orc, golden, func):
    fn = getattr(orc, func)
    for m, truth, _, i in golden_cases(golden, func):
        v = fn(m)
        tol = 1e-10 if abs(truth) > 1e-8 else None
        if tol is None:
            assert abs(v - truth) < 1e-12, (func, i)
        else:
            assert rel_err(v, truth) < tol, (func, i, v, truth)


@pytest.mark.parametrize("func", ["perm", "haf", "lhaf", "tor"])
def test_oracle_quad_matches_mpmath_to_binary128(orc, golden, func):
    fn = getattr(orc, func)
    for m, truth, mp, i in golden_cases(golden, func):
        hi = fn(m, "quad", hilo=True)
        err = abs(complex(hi[0] - mp[0] + (hi[1] - mp[1]), hi[2] - mp[2] + (hi[3] - mp[3])))
        assert err <= 1e-24 * max(abs(truth), 1e-6), (func, i, err)


@pytest.mark.parametrize("func", ["perm", "haf", "lhaf", "tor"])
def test_oracle_fp64_tracks_reference_cpu_fp64(orc, golden, func):
    fn = getattr(orc, func)
    ref = golden[f"{func}_cpu_fp64"]
    for m, truth, _, i in golden_cases(golden, func):
        assert abs(fn(m) - ref[i]) <= 1e-12 * max(abs(truth), 1.0), (func, i)


@pytest.mark.parametrize("func", ["perm", "haf", "lhaf", "tor"])
def test_oracle_indicator_matches_reference(orc, golden, func):
    fn = getattr(orc, func)
    for m, truth, _, i in golden_cases(golden, func):
        _, absn = fn(m, with_absnorm=True)
        ref = golden[f"{func}_absnorm"][i]
        assert absn == pytest.approx(ref, rel=1e-9, abs=1e-14), (func, i)


def test_reference_certified_enclosures_contain_truth(golden):
    for func in ("perm", "haf", "lhaf", "tor"):
        for m, truth, _, i in golden_cases(golden, func):
            v, b = golden[f"{func}_cert_value"][i], golden[f"{func}_cert_bound"][i]
            if np.isfinite(b):
                assert abs(v - truth) <= b, (func, i)


# ---- closed forms --------------------------------------------------------------
@pytest.mark.parametrize("n", range(1, 9))
def test_perm_closed_forms(orc, n):
    assert orc.perm(np.ones((n, n))) == pytest.approx(math.factorial(n), rel=1e-12)
    assert orc.perm(np.eye(n)) == pytest.approx(1.0, abs=1e-12)
    A = np.triu(np.random.default_rng(n).uniform(-1, 1, (n, n)))
    assert orc.perm(A) == pytest.approx(np.prod(np.diag(A)), rel=1e-10, abs=1e-14)


@pytest.mark.parametrize("k", range(1, 6))
def test_haf_closed_forms(orc, k):
    N = 2 * k
    dfact = math.prod(range(1, N, 2))
    assert orc.haf(np.ones((N, N))) == pytest.approx(dfact, rel=1e-12)
    blocks = np.zeros((N, N))
    for j in range(k):
        blocks[2 * j, 2 * j + 1] = blocks[2 * j + 1, 2 * j] = j + 1
    assert orc.haf(blocks) == pytest.approx(math.factorial(k), rel=1e-12)
    assert orc.haf(np.ones((N + 1, N + 1))) == 0


@pytest.mark.parametrize("N", range(1, 9))
def test_lhaf_closed_forms(orc, N):
    telephone = [1, 1, 2, 4, 10, 26, 76, 232, 764]
    assert orc.lhaf(np.ones((N, N))) == pytest.approx(telephone[N], rel=1e-12)
    d = np.arange(2.0, 2.0 + N)
    assert orc.lhaf(np.diag(d)) == pytest.approx(np.prod(d), rel=1e-12)


@pytest.mark.parametrize("a", [0.1, 0.3, 0.6])
@pytest.mark.parametrize("n", [1, 2, 3])
def test_tor_closed_forms(orc, a, n):
    # O = a I (each mode independent): tor = (1/(1-a) - 1)^n = (a/(1-a))^n
    assert orc.tor(a * np.eye(2 * n)) == pytest.approx((a / (1 - a)) ** n, rel=1e-12)
    assert orc.tor(np.zeros((2 * n, 2 * n))) == pytest.approx(0.0, abs=1e-13)


def test_tor_off_domain_is_nan_for_the_real_path(orc):
    O = 2.0 * np.eye(4)  # I - O = -I is not positive definite
    out, _ = orc._call("orc_tor_real", O, 2, 0, real=True)
    assert np.isnan(out[0])


# ---- the reference's own kernels (host build) -----------------------------------
@pytest.mark.parametrize("func", ["perm", "haf", "lhaf", "tor"])
def test_reference_shim_kernels_match_oracle(orc, golden, func):
    if not orc.ref_available():
        pytest.skip("oracle/_ref not built (reference tree absent at build time)")
    by_dim: dict[int, list] = {}
    for m, truth, _, i in golden_cases(golden, func):
        if func == "lhaf" and m.shape[0] % 2:
            continue  # the reference kernel is even-N only (its Python layer augments)
        if func == "tor" and np.any(np.imag(m) != 0):
            continue
        by_dim.setdefault(m.shape[0], []).append((m, truth))
    for d, cases in by_dim.items():
        stack = np.stack([c[0] for c in cases])
        vals = orc.ref_batched(func, stack, "fp64")
        for v, (m, truth) in zip(vals, cases):
            assert abs(v - getattr(orc, func)(m)) <= 1e-11 * max(abs(truth), 1.0)


# ---------------------------------------------------------------- config-size fixture
def test_config_fixture_truths_are_consistent():
    """tests/golden/config_sizes.npz: the binary128 torontonians at 18..24 modes lie
    inside the reference's own certified double-double enclosures (compiled from the
    reference's sources), and the binary64 oracle port stays within its error scale
    N u kappa of the binary128 hafnians and loop hafnians at N = 22..28."""
    from pathlib import Path
    import oracle
    F = dict(np.load(Path(__file__).resolve().parent / "golden" / "config_sizes.npz"))

    def t(q):
        return complex(q[0] + q[1], q[2] + q[3])

    for i, d in enumerate(F["c4_dims"]):
        q = t(F["c4_quad"][i]).real
        assert abs(q - F["c4_ref_value"][i]) <= F["c4_ref_bound"][i] * (1 + 1e-9), (d, q, F["c4_ref_value"][i])
        assert F["c4_ref_bound"][i] <= 1e-11 * abs(q)  # a tight enclosure, not a vacuous one
    for i, f in enumerate(F["c3_funcs"]):
        d = int(F["c3_dims"][i])
        m = F["c3_mats"][i, :d, :d]
        q = t(F["c3_quad"][i])
        v = getattr(oracle, str(f))(m, "fp64")
        kappa = F["c3_absnorm"][i] / abs(q)
        assert abs(v - q) / abs(q) <= 8 * d * 2.0 ** -53 * kappa, (f, d)
