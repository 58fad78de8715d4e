"""The decompositions the torontonian and permanent walks rest on, checked on the CPU.

tor(O) = sum_{S subset [k]} (-1)^(k-|S|) / sqrt(det(I - O)_S)
(cpu_ref/tor_recursive.py:46-100; xxpp indexing: mode i owns rows i and i + k).

The warp walk (gbskernels_b200/csrc/tor_warp.cuh) splits the modes into a prefix
of q = k - r modes, walked by the warp, and a tail of r modes whose 2^r subsets
are the lanes.  At a prefix set S it holds the Schur complement of the whole tail,
Z = M_TT - M_TS M_S^-1 M_ST (M = I - O), and lane T' factors Z restricted to the
modes in T', so that det M_{S u T'} = det M_S * det Z_{T'}.  A lane factors Z
with the rows of excluded modes read from an identity and their pivot reciprocal
set to 0: every term those rows contribute is an exact zero, so the included
entries see exactly the operations of the compressed factorisation.  These tests
check the decomposition against the oracle and that last claim bit for bit.
"""

from __future__ import annotations

import itertools
import math

import numpy as np
import pytest

from gbskernels_b200 import workloads


def _O(k: int, seed: int) -> np.ndarray:
    return workloads.threshold_O(workloads.lossy_squeezed_cov(k, seed=seed))


def _rows(modes, k):
    return [i for i in modes] + [i + k for i in modes]


def _tor_prefix_tail(O: np.ndarray, r: int) -> float:
    k = O.shape[0] // 2
    M = np.eye(2 * k) - O
    q = k - r
    tail = list(range(q, k))
    it = _rows(tail, k)
    total = 0.0
    for m in range(q + 1):
        for S in itertools.combinations(range(q), m):
            iS = _rows(S, k)
            if S:
                MS = M[np.ix_(iS, iS)]
                MST = M[np.ix_(iS, it)]
                Z = M[np.ix_(it, it)] - MST.T @ np.linalg.solve(MS, MST)
                dS = np.linalg.det(MS)
            else:
                Z, dS = M[np.ix_(it, it)], 1.0
            for mt in range(r + 1):
                for T in itertools.combinations(range(r), mt):
                    sel = _rows(T, r)
                    dT = np.linalg.det(Z[np.ix_(sel, sel)]) if T else 1.0
                    total += (-1) ** (k - m - mt) / math.sqrt(dS * dT)
    return total


@pytest.mark.parametrize("k,r", [(4, 2), (6, 3), (7, 5), (8, 5)])
def test_prefix_times_tail_schur_complement_is_the_torontonian(orc, k, r):
    O = _O(k, seed=20 + k)
    ref = orc.tor(O)
    got = _tor_prefix_tail(O, r)
    assert abs(got - ref) <= 1e-11 * max(abs(ref), 1.0)


def _chol_logdet_terms(Z: np.ndarray, include: list[bool]):
    """Left-looking Cholesky in a fixed scalar order; rows with include False are
    read from an identity and get pivot reciprocal 0.  Returns the pivots of the
    included rows and the factor."""
    n = Z.shape[0]
    Zp = Z.copy()
    for i in range(n):
        if not include[i]:
            Zp[i, :] = 0.0
            Zp[:, i] = 0.0
            Zp[i, i] = 1.0
    L = np.zeros((n, n))
    piv = []
    for j in range(n):
        s = float(Zp[j, j])
        for t in range(j):
            s = s - L[j, t] * L[j, t]
        p = math.sqrt(s)
        rinv = 1.0 / p if include[j] else 0.0
        L[j, j] = p
        if include[j]:
            piv.append(p)
        for i in range(j + 1, n):
            x = float(Zp[i, j])
            for t in range(j):
                x = x - L[i, t] * L[j, t]
            L[i, j] = x * rinv
    return piv, L


@pytest.mark.parametrize("r", [3, 5])
def test_packed_identity_rows_reproduce_the_compressed_factor_bit_for_bit(r):
    k = r + 3
    O = _O(k, seed=40 + r)
    M = np.eye(2 * k) - O
    it = _rows(range(k - r, k), k)
    Z = M[np.ix_(it, it)]  # the tail block at the empty prefix (any SPD block will do)
    for mt in range(r + 1):
        for T in itertools.combinations(range(r), mt):
            inc_modes = set(T)
            include = [(i % r) in inc_modes for i in range(2 * r)]
            piv_p, L_p = _chol_logdet_terms(Z, include)
            sel = [i for i in range(2 * r) if include[i]]
            piv_c, L_c = _chol_logdet_terms(Z[np.ix_(sel, sel)], [True] * len(sel))
            assert [x.hex() for x in piv_p] == [x.hex() for x in piv_c]
            sub = L_p[np.ix_(sel, sel)]
            assert np.array_equal(sub.view(np.uint64), L_c.view(np.uint64))


# ---------------------------------------------------------------- permanent
# The Glynn walk (gbskernels_b200/csrc/perm_tor.cuh) gives each lane an aligned
# range [i0, i0 + R) of Gray indices: it starts from the row sums at delta(gray(i0))
# and then flips column ctz(j) + 1 at step j, with the sign of the flip read from
# gray(i0 + j).  Because i0 is a multiple of R, ctz(i0 + j) = ctz(j): every lane of
# a warp flips the same column at the same step.


def _gray(i: int) -> int:
    return i ^ (i >> 1)


def _lane_range(A: np.ndarray, i0: int, R: int) -> complex:
    n = A.shape[0]
    g0 = _gray(i0)
    delta = np.array([1.0] + [(-1.0 if (g0 >> (c - 1)) & 1 else 1.0) for c in range(1, n)])
    rs = A @ delta
    sign = -1.0 if i0 & 1 else 1.0
    acc = sign * np.prod(rs)
    for j in range(1, R):
        i = i0 + j
        k = (j & -j).bit_length() - 1
        assert k == (i & -i).bit_length() - 1  # the same column in every lane
        step = -2.0 if (_gray(i) >> k) & 1 else 2.0
        rs = rs + step * A[:, k + 1]
        sign = -sign
        acc += sign * np.prod(rs)
    return acc


@pytest.mark.parametrize("n,rlog", [(3, 1), (5, 2), (7, 3), (8, 0)])
def test_aligned_gray_ranges_sum_to_the_permanent(orc, n, rlog):
    rng = np.random.default_rng(60 + n)
    A = rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))
    terms = 1 << (n - 1)
    R = 1 << min(rlog, n - 1)
    total = sum(_lane_range(A, i0, R) for i0 in range(0, terms, R))
    got = total / terms
    ref = orc.perm(A)
    assert abs(got - ref) <= 1e-12 * max(abs(ref), 1.0)
