"""Seeded synthetic inputs with the shapes, sizes and value distributions of the
benchmark configurations (no datasets are involved; every matrix is generated).

Constructions (standard, re-implemented here):
  * Haar-random unitary: QR of a complex Ginibre matrix with the phases of diag(R)
    divided out (Mezzadri 2007) -- as the reference's bench/_inputs.py:242-249.
  * Pure-state GBS kernel A = U diag(tanh r) U^T (sampling/gbs.py:40-64), photon
    pattern -> index list with repeats -> A[idx][:, idx]; loop weights gamma on the
    diagonal for the loop hafnian (sampling/gbs.py:131-139).
  * Threshold-detector matrix O_x = I - Sigma_x^{-1} in xxpp ordering of a lossy
    squeezed state, Sigma_x = (cov + I)/2 (sampling/gbs.py:241-275), restricted to a
    click pattern S as O_x[[S, S+M]][:, [S, S+M]].
"""

from __future__ import annotations

import numpy as np


def haar_unitary(m: int, rng: np.random.Generator) -> np.ndarray:
    z = (rng.standard_normal((m, m)) + 1j * rng.standard_normal((m, m))) / np.sqrt(2.0)
    q, r = np.linalg.qr(z)
    ph = np.diagonal(r).copy()
    ph /= np.abs(ph)
    return q * ph


# ---------------------------------------------------------------- config 1
def haf_real_batch(B: int = 4096, N: int = 16, seed: int = 1) -> np.ndarray:
    """B real symmetric N x N matrices A = (G + G^T)/sqrt(2), G iid N(0, 1)."""
    rng = np.random.default_rng(seed)
    G = rng.standard_normal((B, N, N))
    return (G + np.transpose(G, (0, 2, 1))) / np.sqrt(2.0)


# ---------------------------------------------------------------- config 2
def perm_haar_batch(B: int = 1024, n: int = 20, M: int = 400, seed: int = 2) -> np.ndarray:
    """B complex n x n submatrices of a Haar M x M unitary: rows = n distinct random
    modes (the detected outputs), columns = modes 0..n-1 (the input photons)."""
    rng = np.random.default_rng(seed)
    U = haar_unitary(M, rng)
    out = np.empty((B, n, n), dtype=np.complex128)
    cols = np.arange(n)
    for b in range(B):
        rows = rng.choice(M, size=n, replace=False)
        out[b] = U[np.ix_(rows, cols)]
    return out


# ---------------------------------------------------------------- config 3
def gbs_kernel(M: int = 100, r: float = 1.0, seed: int = 3) -> np.ndarray:
    rng = np.random.default_rng(seed)
    U = haar_unitary(M, rng)
    return U @ np.diag(np.full(M, np.tanh(r))) @ U.T


def mixed_haf_lhaf(B: int = 65536, sizes=tuple(range(8, 29, 2)), M: int = 100, seed: int = 3,
                   gamma_var: float = 0.1):
    """The persistent mixed-size batch: B complex instances, N uniform over `sizes`,
    function 50/50 haf / lhaf; each a submatrix of A = U diag(tanh 1) U^T with the
    repeated rows / columns of a random photon pattern with N photons over M modes;
    loop weights gamma_i ~ CN(0, gamma_var) on the loop-hafnian diagonals.
    Returns (funcs, mats)."""
    rng = np.random.default_rng(seed)
    A = gbs_kernel(M, 1.0, seed)
    gamma = (rng.standard_normal(M) + 1j * rng.standard_normal(M)) * np.sqrt(gamma_var / 2.0)
    Ns = rng.choice(np.asarray(sizes), size=B)
    is_loop = rng.random(B) < 0.5
    funcs, mats = [], []
    for b in range(B):
        N = int(Ns[b])
        idx = np.sort(rng.integers(0, M, size=N))   # photon pattern with repeats
        S = np.ascontiguousarray(A[np.ix_(idx, idx)])
        if is_loop[b]:
            S = S.copy()
            np.fill_diagonal(S, gamma[idx])
            funcs.append("lhaf")
        else:
            funcs.append("haf")
        mats.append(S)
    return funcs, mats


# ---------------------------------------------------------------- config 4
def lossy_squeezed_cov(M: int = 50, rlo: float = 0.5, rhi: float = 1.2, eta: float = 0.7,
                       seed: int = 4) -> np.ndarray:
    """xxpp covariance (hbar = 2) of M single-mode squeezers through a Haar
    interferometer followed by uniform loss of transmission eta."""
    rng = np.random.default_rng(seed)
    r = rng.uniform(rlo, rhi, M)
    U = haar_unitary(M, rng)
    sq = np.diag(np.concatenate([np.exp(-2 * r), np.exp(2 * r)]))
    O = np.block([[U.real, -U.imag], [U.imag, U.real]])
    pure = O @ sq @ O.T
    return eta * pure + (1.0 - eta) * np.eye(2 * M)


def threshold_O(cov: np.ndarray) -> np.ndarray:
    n2 = cov.shape[0]
    Sx = (cov + np.eye(n2)) / 2.0
    Sx = (Sx + Sx.T) / 2.0
    Ox = np.eye(n2) - np.linalg.inv(Sx)
    return np.ascontiguousarray((Ox + Ox.T) / 2.0)


def tor_click_batch(B: int = 8192, kmin: int = 10, kmax: int = 24, M: int = 50, seed: int = 4):
    """B real O_S (2k x 2k, xxpp) for click patterns of k uniform in [kmin, kmax]."""
    rng = np.random.default_rng(seed + 1)
    Ox = threshold_O(lossy_squeezed_cov(M, seed=seed))
    ks = rng.integers(kmin, kmax + 1, size=B)
    mats = []
    for b in range(B):
        S = np.sort(rng.choice(M, size=int(ks[b]), replace=False))
        idx = np.concatenate([S, S + M])
        mats.append(np.ascontiguousarray(Ox[np.ix_(idx, idx)]))
    return mats


# ---------------------------------------------------------------- config 5
def serving_chains(n_req: int, rate: float, seed: int = 5, M: int = 50, nmin: int = 6, nmax: int = 30,
                   lanes: int = 8):
    """Poisson arrivals of chain-rule sampler queries on resident states.

    States: the pure-state GBS kernel A = U diag(tanh 1) U^T (M x M) with loop
    weights gamma ~ CN(0, 0.1), and the threshold-detector matrix O_x (2M x 2M, xxpp)
    of a lossy squeezed state.  `lanes` samplers run side by side; each runs chains
    one after another, and a chain is the sequence of growing submatrices a
    chain-rule sampler evaluates as it extends its pattern: for haf / lhaf the
    prefixes of a sorted photon pattern (repeated modes; two photons more per step,
    sizes up to n_final uniform over the even values in [nmin, nmax]), for tor the
    click-set prefixes (one mode more per step, matrix side 2k).  Arrival i is the
    next query of lane i mod `lanes`.  Precision per query: fp64 70 % / auto 20 % /
    certified 10 %.

    Returns (states, queries): states = {"A": A, "gamma": gamma, "O": O_x};
    queries = [(arrival_s, func, precision, state_key, idx, use_gamma)], the matrix
    of a query being state[idx][:, idx] (with gamma[idx] on the diagonal when
    use_gamma)."""
    rng = np.random.default_rng(seed)
    A = gbs_kernel(M, 1.0, seed)
    gamma = (rng.standard_normal(M) + 1j * rng.standard_normal(M)) * np.sqrt(0.05)
    Ox = threshold_O(lossy_squeezed_cov(M, seed=seed))
    t = np.cumsum(rng.exponential(1.0 / rate, size=n_req))
    sizes = np.arange(nmin, nmax + 1, 2)

    def new_chain():
        func = ["haf", "lhaf", "tor"][int(rng.integers(0, 3))]
        steps = int(rng.integers(1, 5))
        nf = int(rng.choice(sizes))
        if func == "tor":
            kf = nf // 2
            S = np.sort(rng.choice(M, size=kf, replace=False))
            k0 = max(nmin // 2, kf - steps + 1)
            return [(func, "O", np.concatenate([S[:k], S[:k] + M]).astype(np.int32), False)
                    for k in range(k0, kf + 1)]
        idx = np.sort(rng.integers(0, M, size=nf)).astype(np.int32)
        n0 = max(nmin, nf - 2 * (steps - 1))
        return [(func, "A", idx[:n].copy(), func == "lhaf") for n in range(n0, nf + 1, 2)]

    pending = [[] for _ in range(lanes)]
    queries = []
    for i in range(n_req):
        lane = i % lanes
        if not pending[lane]:
            pending[lane] = new_chain()
        func, key, idx, ug = pending[lane].pop(0)
        u = rng.random()
        prec = "fp64" if u < 0.7 else ("auto" if u < 0.9 else "certified")
        queries.append((float(t[i]), func, prec, key, idx, ug))
    return {"A": A, "gamma": gamma, "O": Ox}, queries


def gather_query(states: dict, key: str, idx: np.ndarray, use_gamma: bool) -> np.ndarray:
    """The matrix of a resident-state query, gathered on the host: state[idx][:, idx]
    (gamma[idx] on the diagonal when use_gamma), complex128."""
    S = np.ascontiguousarray(np.asarray(states[key], dtype=np.complex128)[np.ix_(idx, idx)])
    if use_gamma:
        np.fill_diagonal(S, states["gamma"][idx])
    return S


def serving_stream(n_req: int, rate: float, seed: int = 5, M: int = 50, nmin: int = 6, nmax: int = 30):
    """The chain-rule query stream of `serving_chains` with every matrix gathered on
    the host: [(arrival_s, func, precision, matrix)] (the host-matrix form of the
    same requests, for servers fed explicit matrices and for offline batches)."""
    states, queries = serving_chains(n_req, rate, seed=seed, M=M, nmin=nmin, nmax=nmax)
    return [(ta, f, p, gather_query(states, k, idx, ug)) for (ta, f, p, k, idx, ug) in queries]


# ---------------------------------------------------------------- algorithmic work
def ref_flops(func: str, dim: int, real: bool = False) -> float:
    """Algorithmic FP64 flops of the REFERENCE algorithm for one instance (complex
    MAC = 8 flops, real MAC = 2):
      haf:  (n-1) n^2 (n+3) 2^n MACs, n = N/2 (power trace, n-1 products per subset)
      lhaf: haf + n (s^2 + s) per subset  ~ haf + 2^n n (4n^2/2 + ...)  (loop matvecs)
      perm: 2^(n-1) (10 n - 4) flops (Glynn Gray walk)
      tor:  2 * 2^k (k^2 - k + 1) flops, k = modes (prefix Cholesky appends + leaves)."""
    if func in ("haf", "lhaf"):
        n = dim // 2 + (dim & 1 if func == "lhaf" else 0)
        macs = (n - 1) * n * n * (n + 3) * 2.0 ** n
        if func == "lhaf":
            # loop term: one s x s matvec per power k = 1..n, sum_m C(n,m) (2m)^2 n
            macs += n * (4.0 * n * (n + 1) * 2.0 ** (n - 2))
        return macs * (2.0 if real else 8.0)
    if func == "perm":
        return 2.0 ** (dim - 1) * (10 * dim - 4)
    if func == "tor":
        k = dim // 2
        return 2.0 * 2.0 ** k * (k * k - k + 1)
    raise ValueError(func)
