"""The decompositions the torontonian, permanent and sieve walks and the subset LU
rest on, checked on the CPU.

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


# ---------------------------------------------------------------- repeated-row sieve
# The sieve kernel (gbskernels_b200/csrc/k_sieve.cu) walks the digit vectors v of a
# repetition pattern in reflected mixed-radix Gray order (digit 0 fastest, the
# largest n_i on top with only floor(n_top / 2) + 1 values: the v <-> n - v
# symmetry, weight 2 below the middle).  A work item restarts at Gray index t0 from
# a directly decoded state: per digit q = t0 / place, b = q mod radix, reflected
# (g = radix - 1 - b) when the parity of q / radix is odd, the top digit never
# reflected.  A step moves the lowest digit that is not at the end of its run by
# +-1 (the sign from its reflection parity) and resets the digits below it.


def _sieve_digits(reps):
    modes = [i for i, n in enumerate(reps) if n > 0]
    modes.sort(key=lambda i: reps[i])  # largest n_i on top (last digit)
    ns = [int(reps[i]) for i in modes]
    radix = [n + 1 for n in ns]
    radix[-1] = ns[-1] // 2 + 1
    place = [1]
    for r in radix[:-1]:
        place.append(place[-1] * r)
    return modes, ns, radix, place, place[-1] * radix[-1]


def _decode(t, radix, place):
    nd = len(radix)
    b, par, g = [], [], []
    for i in range(nd):
        q = t // place[i]
        bi = q % radix[i]
        pi = 0 if i == nd - 1 else (q // radix[i]) & 1
        b.append(bi)
        par.append(pi)
        g.append(radix[i] - 1 - bi if pi else bi)
    return b, par, g


def _step(b, par, g, radix):
    j = next(i for i in range(len(radix)) if b[i] < radix[i] - 1)
    d = -1 if par[j] else 1
    for i in range(j):
        b[i] = 0
        par[i] ^= 1
    b[j] += 1
    g[j] += d
    return j, d


@pytest.mark.parametrize("reps", [[3], [2, 1], [1, 2, 3], [2, 2, 2, 1], [4, 1, 0, 3]])
def test_sieve_gray_walk_decodes_steps_and_covers(reps):
    modes, ns, radix, place, terms = _sieve_digits(reps)
    seen = set()
    b, par, g = _decode(0, radix, place)
    for t in range(terms):
        assert (b, par, g) == _decode(t, radix, place)  # a restart anywhere agrees
        seen.add(tuple(g))
        if t + 1 < terms:
            prev = list(g)
            _step(b, par, g, radix)
            diff = [abs(x - y) for x, y in zip(g, prev)]
            assert sum(diff) == 1  # one digit, by one
    assert len(seen) == terms  # every digit vector of the halved box exactly once
    assert all(0 <= gi <= (n if i < len(ns) - 1 else n // 2) for gi_vec in seen
               for i, (gi, n) in enumerate(zip(gi_vec, ns)))


def _sieve_value(A, gamma, reps):
    modes, ns, radix, place, terms = _sieve_digits(reps)
    N = sum(ns)
    K = N // 2
    Am = A[np.ix_(modes, modes)]
    gm = np.asarray(gamma)[modes]
    tot = 0j
    b, par, g = _decode(0, radix, place)
    for t in range(terms):
        x = np.array([n - 2 * gi for n, gi in zip(ns, g)], dtype=float)
        s2 = x @ Am @ x
        mu = x @ gm
        sn = sum(math.comb(N, 2 * k) * math.prod(range(1, 2 * k, 2)) * s2 ** k * mu ** (N - 2 * k)
                 for k in range(K + 1))
        w = 2.0 if 2 * g[-1] < ns[-1] else 1.0
        sgn = -1.0 if sum(g) & 1 else 1.0
        tot += sgn * w * math.prod(math.comb(n, gi) for n, gi in zip(ns, g)) * sn
        if t + 1 < terms:
            _step(b, par, g, radix)
    return tot / (math.factorial(N) * 2 ** N)


@pytest.mark.parametrize("reps", [[2, 1, 1], [1, 2, 3], [2, 2, 0, 2], [3, 1, 2, 2]])
def test_sieve_gray_walk_value_equals_the_oracle(orc, reps):
    rng = np.random.default_rng(sum(reps) * 7 + len(reps))
    M = len(reps)
    G = rng.standard_normal((M, M)) + 1j * rng.standard_normal((M, M))
    A = (G + G.T) / 2
    gamma = (rng.standard_normal(M) + 1j * rng.standard_normal(M)) * 0.3
    got = _sieve_value(A, gamma, reps)
    ref = orc.lhaf_repeated(A, gamma, np.asarray(reps))
    assert abs(got - ref) <= 1e-10 * max(abs(ref), 1.0)


# ---------------------------------------------------------------- complex torontonian
# The subset LU of a complex minor (gbskernels_b200/csrc/tor_lu.cuh) never moves a
# row: at column c the pivot is the unused row of largest |M[r][c]|^2 (ties: the
# lowest), and the permutation's parity is accumulated as the number of unused rows
# below the pivot row, step by step (those are exactly the inversions the pivot
# contributes).  det = (-1)^parity * prod pivots.


def _det_no_swap(M: np.ndarray) -> complex:
    M = M.astype(np.complex128).copy()
    m = M.shape[0]
    used = [False] * m
    det = 1.0 + 0j
    inversions = 0
    for c in range(m):
        cand = [(abs(M[r, c]) ** 2, -r) for r in range(m) if not used[r]]
        best, negwho = max(cand)
        who = -negwho
        if not best > 0:
            return 0j
        inversions += sum(1 for r in range(who) if not used[r])
        piv = M[who, c]
        det *= piv
        used[who] = True
        for r in range(m):
            if not used[r]:
                f = M[r, c] / piv
                M[r, c + 1:] -= f * M[who, c + 1:]
    return -det if inversions & 1 else det


@pytest.mark.parametrize("m", [1, 2, 5, 8, 12])
def test_lu_without_row_moves_gives_the_determinant(m):
    rng = np.random.default_rng(80 + m)
    for trial in range(20):
        A = rng.standard_normal((m, m)) + 1j * rng.standard_normal((m, m))
        if trial % 4 == 0 and m > 1:
            A[:, 0] = A[0, 0]  # ties in the first pivot column
        ref = np.linalg.det(A)
        assert abs(_det_no_swap(A) - ref) <= 1e-10 * max(abs(ref), 1.0)
