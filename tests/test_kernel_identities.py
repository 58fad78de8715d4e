"""The algebra the hafnian kernel rests on, checked on the CPU against the oracle.

The reference evaluates each subset term from the n - 1 powers C, C^2, ..., C^n
(cpu_ref/hafnian.py:83-93, cpu_ref/loop_hafnian.py:94-104).  The tensor-core
kernel (gbskernels_b200/csrc/haf_pt.cuh) computes only C, ..., C^h with
h = ceil(n / 2) and reads every trace and loop term off those powers:

  tr(C^{2a})   = sum_{i,t} C^a[i][t] C^a[i^1][t^1]
  tr(C^{2a-1}) = sum_{i,t} C^a[i][t] C^{a-1}[i^1][t^1]
  d^T X C^{k-1} d = sum_i y_a[i^1] y_b[i],   y_a = C^a d,  a + b = k - 1,

all three from C^T = X C X (C = B_S X with B_S symmetric).  In the mma
accumulator layout the partner (i^1, t^1) of a lane's element sits in lane ^ 5,
same register.  These tests restate the kernel's formulation in numpy and check
it against the direct formula and against the oracle's hafnians.
"""

from __future__ import annotations

import numpy as np
import pytest


def _subset_C(A: np.ndarray, mask: int, n: int, loop: bool):
    """C = B_S X and d = diag(B_S) for the pairs in `mask` (the kernel's staging)."""
    idx = [2 * i + b for i in range(n) if (mask >> i) & 1 for b in (0, 1)]
    s = len(idx)
    C = np.empty((s, s), dtype=np.complex128)
    for r in range(s):
        for c in range(s):
            rr, cc = idx[r], idx[c ^ 1]
            C[r, c] = A[rr, cc] if (loop or rr != cc) else 0.0
    d = np.array([A[i, i] for i in idx], dtype=np.complex128)
    return C, d


def _partner(M: np.ndarray) -> np.ndarray:
    """M[i^1][t^1] as a matrix."""
    p = np.arange(M.shape[0]) ^ 1
    return M[np.ix_(p, p)]


def _kg_half_powers(C: np.ndarray, d: np.ndarray, n: int, loop: bool) -> np.ndarray:
    """k g_k, k = 1..n, from the powers C^0..C^h only (the kernel's formulation)."""
    s = C.shape[0]
    h = (n + 1) // 2
    pw = [np.eye(s, dtype=np.complex128)]
    for _ in range(h):
        pw.append(pw[-1] @ C)
    p = np.zeros(n + 1, dtype=np.complex128)
    for a in range(1, h + 1):
        if 2 * a - 1 <= n:
            p[2 * a - 1] = np.sum(pw[a] * _partner(pw[a - 1]))
        if 2 * a <= n:
            p[2 * a] = np.sum(pw[a] * _partner(pw[a]))
    kg = p / 2
    if loop:
        y = [pw[a] @ d for a in range(h + 1)]
        xs = np.arange(s) ^ 1
        for k in range(1, n + 1):
            aa = (k - 1) >> 1
            bb = k - 1 - aa
            kg[k] += k * 0.5 * np.sum(y[aa][xs] * y[bb])
    return kg


def _kg_direct(C: np.ndarray, d: np.ndarray, n: int, loop: bool) -> np.ndarray:
    """k g_k from tr(C^k) and d^T X C^{k-1} d (the reference's formulation)."""
    s = C.shape[0]
    X = np.zeros((s, s))
    X[np.arange(s), np.arange(s) ^ 1] = 1.0
    kg = np.zeros(n + 1, dtype=np.complex128)
    P = np.eye(s, dtype=np.complex128)
    for k in range(1, n + 1):
        Q = P
        P = P @ C
        kg[k] = np.trace(P) / 2
        if loop:
            kg[k] += k * 0.5 * (d @ X @ Q @ d)
    return kg


def _newton(kg: np.ndarray, n: int) -> complex:
    e = [1.0 + 0j]
    for j in range(1, n + 1):
        e.append(sum(kg[k] * e[j - k] for k in range(1, j + 1)) / j)
    return e[n]


def _sym(rng, N):
    G = rng.standard_normal((N, N)) + 1j * rng.standard_normal((N, N))
    return (G + G.T) / 2


@pytest.mark.parametrize("N", [2, 4, 6, 8, 10])
@pytest.mark.parametrize("loop", [False, True])
def test_half_powers_give_every_trace_and_loop_term(N, loop):
    rng = np.random.default_rng(100 + N + 7 * loop)
    A = _sym(rng, N)
    n = N // 2
    for mask in range(1, 1 << n):
        C, d = _subset_C(A, mask, n, loop)
        np.testing.assert_allclose(C.T, _partner(C), rtol=0, atol=0)  # C^T = X C X
        a = _kg_half_powers(C, d, n, loop)
        b = _kg_direct(C, d, n, loop)
        np.testing.assert_allclose(a[1:], b[1:], rtol=1e-12, atol=1e-12 * np.abs(b[1:]).max())


@pytest.mark.parametrize("N", [4, 8, 12])
@pytest.mark.parametrize("func", ["haf", "lhaf"])
def test_half_powers_hafnian_equals_the_oracle(orc, N, func):
    rng = np.random.default_rng(7 * N + (func == "lhaf"))
    A = _sym(rng, N)
    loop = func == "lhaf"
    n = N // 2
    total = 0j
    for mask in range(1 << n):
        m = bin(mask).count("1")
        if m == 0:
            continue  # [lambda^n] exp(0) = 0 for n >= 1
        C, d = _subset_C(A, mask, n, loop)
        t = _newton(_kg_half_powers(C, d, n, loop), n)
        total += -t if (n - m) & 1 else t
    ref = getattr(orc, func)(A)
    assert abs(total - ref) <= 1e-11 * max(abs(ref), 1.0)


def test_partner_element_is_lane_xor_5():
    """Accumulator layout of mma.m16n8k8 .f64 over the interleaved real embedding:
    lane = 4 g + t4 holds complex element (row g, column 4 nt + t4) in registers
    0..1 and (row g + 8, same column) in registers 2..3.  The partner (i^1, t^1)
    of every element is held by lane ^ 5 in the same registers."""
    def owner(row, col):
        nt, t4 = divmod(col, 4)
        g, hi = row % 8, row >= 8
        return 4 * g + t4, nt, hi
    for row in range(16):
        for col in range(32):
            lane, nt, hi = owner(row, col)
            plane, pnt, phi = owner(row ^ 1, col ^ 1)
            assert (plane, pnt, phi) == (lane ^ 5, nt, hi)
