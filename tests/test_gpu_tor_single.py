"""Single-large torontonian (one instance over the whole GPU, up to 32 modes)
against the binary128 oracle at small sizes and, past the batched cap, through the
direct-sum identity tor(O1 (+) O2) = tor(O1) tor(O2) with the halves evaluated by
the independent double-double kernel.  Reference test model:
tests/test_torontonian.py (single-large rows) and tests/test_certified.py."""

from __future__ import annotations

import numpy as np
import pytest

from conftest import rel_err

pytestmark = pytest.mark.gpu
RNG = np.random.default_rng(31)


def phys_O(n):
    X = RNG.standard_normal((2 * n, 2 * n))
    S = X @ X.T / (2 * n) + np.eye(2 * n)
    O = np.eye(2 * n) - np.linalg.inv(S)
    return (O + O.T) / 2


def direct_sum(O1, O2):
    n1, n2 = O1.shape[0] // 2, O2.shape[0] // 2
    n = n1 + n2
    O = np.zeros((2 * n, 2 * n))
    i1 = np.r_[0:n1, n:n + n1]
    i2 = np.r_[n1:n, n + n1:2 * n]
    O[np.ix_(i1, i1)] = O1
    O[np.ix_(i2, i2)] = O2
    return O


@pytest.mark.parametrize("n,groups", [(3, None), (8, 0), (10, 10), (12, None)])
def test_tor_single_vs_binary128(gpu, orc, n, groups):
    O = phys_O(n)
    truth = orc.tor(O, "quad").real
    _, kd = gpu.tor_batched(O[None], precision="auto", return_diagnostics=True)
    kappa = kd[0]["cancellation"]  # sum |term| / |tor|
    v = gpu.tor_single(O, groups=groups)
    assert rel_err(v, truth) < max(1e-13, 1e-15 * kappa)
    vc, d = gpu.tor_single(O, groups=groups, certified=True)
    assert vc == v
    assert abs(vc - truth) <= d["abs_error_bound"]
    assert d["rel_error_bound"] < 1e-9 * kappa
    assert d["tier"] == "certified-fp64"


@pytest.mark.parametrize("n1,n2", [(13, 13), (16, 16)])
def test_tor_single_direct_sum_past_the_batched_cap(gpu, n1, n2):
    O1, O2 = phys_O(n1), phys_O(n2)
    O = direct_sum(O1, O2)
    halves = gpu.tor_batched(np.stack([O1, O2]) if n1 == n2 else [O1, O2], precision="dd")
    want = (halves[0] * halves[1]).real
    _, kd = gpu.tor_batched(O1[None], precision="auto", return_diagnostics=True)
    v = gpu.tor_single(O)
    # the cancellation of the product grows like the product of the halves'
    assert rel_err(v, want) < max(1e-10, 1e-15 * kd[0]["cancellation"] ** 2)
    vc, d = gpu.tor_single(O, certified=True)
    assert vc == v
    assert abs(vc - want) <= d["abs_error_bound"] + 1e-15 * abs(want)


def test_tor_single_off_domain_raises(gpu):
    with pytest.raises(ValueError, match="physical domain"):
        gpu.tor_single(1.5 * np.eye(8))
    with pytest.raises(ValueError):
        gpu.tor_single(1.5 * np.eye(8), certified=True)
    with pytest.raises(ValueError):
        gpu.tor_single(1.5 * np.eye(8), dd=True)


@pytest.mark.parametrize("n", [6, 12])
def test_tor_single_dd_certified(gpu, orc, n):
    O = phys_O(n)
    truth = orc.tor(O, "quad").real
    v, d = gpu.tor_single(O, dd=True)
    assert d["tier"] == "certified-dd"
    assert abs(v - truth) <= d["abs_error_bound"] + 1e-30
    assert d["rel_error_bound"] < 1e-13
