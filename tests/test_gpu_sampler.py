"""Resident sampler chain (on-device conditional draw): the device-gathered
conditional hafnians against the binary128 oracle on the same index rule, and the
drawn distribution against the exact per-mode-truncated chain distribution
computed on the host (reference test model: core/check_sampler_*.cu and
tests/test_sampler.py -- distributional, since cuRAND streams differ from numpy's)."""

from __future__ import annotations

import itertools
from math import factorial

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _cov(M, seed=1):
    from gbskernels_b200 import workloads
    return workloads.lossy_squeezed_cov(M, rlo=0.4, rhi=0.8, eta=0.8, seed=seed)


def _index(prefix, j, k):
    idx = [i for i in range(k - 1) for _ in range(prefix[i])] + [k - 1] * j
    idx += [i + k for i in range(k - 1) for _ in range(prefix[i])] + [2 * k - 1] * j
    return idx


def _weights_host(orc, A, prefix, k, cutoff):
    out = []
    for j in range(cutoff + 1):
        idx = _index(prefix, j, k)
        out.append(1.0 if not idx else orc.haf(A[np.ix_(idx, idx)], "quad").real)
    return np.array(out)


def test_conditional_weights_vs_oracle(gpu, orc):
    from gbskernels_b200 import sampler
    M, cutoff = 3, 4
    cov = _cov(M)
    rng = np.random.default_rng(5)
    for k in (1, 2, 3):
        A = sampler.reduced_A(cov, k)
        pre = rng.integers(0, cutoff + 1, (6, max(k - 1, 1)))[:, :k - 1]
        w = sampler.conditional_weights(cov, k, pre, cutoff)
        for r in range(len(pre)):
            want = _weights_host(orc, A, pre[r], k, cutoff)
            scale = np.maximum(np.abs(want), 1e-300)
            assert np.all(np.abs(w[r] - want) <= 1e-10 * scale + 1e-15), (k, r, w[r], want)


def _chain_distribution(orc, cov, cutoff):
    from gbskernels_b200 import sampler
    M = cov.shape[0] // 2
    As = [sampler.reduced_A(cov, k) for k in range(1, M + 1)]
    invf = np.array([1.0 / factorial(j) for j in range(cutoff + 1)])
    P = {}
    for out in itertools.product(range(cutoff + 1), repeat=M):
        p = 1.0
        for k in range(1, M + 1):
            w = np.maximum(_weights_host(orc, As[k - 1], out[:k - 1], k, cutoff), 0.0) * invf
            s = w.sum()
            p *= (1.0 if out[k - 1] == 0 else 0.0) if s <= 0 else w[out[k - 1]] / s
            if p == 0.0:
                break
        P[out] = p
    return P


def test_drawn_distribution_matches_the_chain(gpu, orc):
    from gbskernels_b200 import sampler
    M, cutoff, S = 2, 4, 40000
    cov = _cov(M, seed=3)
    samples = sampler.sample_resident(cov, S, cutoff=cutoff, seed=11)
    assert samples.shape == (S, M) and samples.min() >= 0 and samples.max() <= cutoff
    P = _chain_distribution(orc, cov, cutoff)
    assert abs(sum(P.values()) - 1.0) < 1e-12
    emp = {}
    for row in map(tuple, samples):
        emp[row] = emp.get(row, 0) + 1
    tv = 0.5 * sum(abs(emp.get(o, 0) / S - p) for o, p in P.items())
    tv += 0.5 * sum(c / S for o, c in emp.items() if o not in P)
    assert tv < 0.02, tv


def test_seeds_and_edge_cases(gpu):
    from gbskernels_b200 import sampler
    cov = _cov(3, seed=2)
    a = sampler.sample_resident(cov, 500, cutoff=3, seed=7)
    b = sampler.sample_resident(cov, 500, cutoff=3, seed=7)
    c = sampler.sample_resident(cov, 500, cutoff=3, seed=8)
    assert np.array_equal(a, b) and not np.array_equal(a, c)
    assert sampler.sample_resident(cov, 0, cutoff=3).shape == (0, 3)
    vac = np.eye(4)  # vacuum: every count is 0
    assert np.all(sampler.sample_resident(vac, 100, cutoff=4, seed=1) == 0)
    with pytest.raises(ValueError):
        sampler.sample_resident(_cov(5), 10, cutoff=4)  # 2 M cutoff = 40 > 32


@pytest.mark.parametrize("M,cutoff,S", [(8, 2, 20000), (4, 4, 20000), (16, 1, 5000), (2, 8, 3000)])
def test_prefix_sharing_gives_the_same_samples(gpu, lib, M, cutoff, S):
    """Draws that share a prefix share their conditional hafnians (evaluated once per
    distinct prefix): the samples equal, count for count, those of evaluating every
    draw's conditionals separately, with the same seed."""
    from gbskernels_b200 import sampler
    cov = _cov(M, seed=5)
    try:
        lib.gbs_sampler_set_dedup(0)
        plain = sampler.sample_resident(cov, S, cutoff=cutoff, seed=21)
    finally:
        lib.gbs_sampler_set_dedup(1)
    shared = sampler.sample_resident(cov, S, cutoff=cutoff, seed=21)
    assert np.array_equal(shared, plain)
    assert shared.sum() > 0
