"""On-device conditional draw: the resident sampler chain.

``sample_resident(cov, num_samples, cutoff)`` draws photon-number samples of a
zero-displacement Gaussian state from the sequentially per-mode-truncated
chain-rule distribution: mode k's count is drawn from
P(n_k = j | prefix) proportional to max(Re haf(A_k[idx, idx]), 0) / j!, j = 0..cutoff,
with A_k the A-matrix of the state reduced to modes 1..k and idx the prefix
photons (and j) repeated on both the a and a-dagger blocks.  Everything after the
A_k (computed here once, on the host) runs on the device: per mode one gather of
the conditional submatrices, one work-item launch of their hafnians, one draw
(inverse CDF, one Philox uniform per draw and mode); the counts are read back at
the end.  Reference: sampling/sampler.py:86-92 (A_k), :214-244 (the resident
path), core/sampler_session.cu:66-137.  cuRAND streams differ from numpy's, so
samples agree with a host sampler in distribution, not draw by draw.
"""

from __future__ import annotations

from math import factorial

import numpy as np

from . import _lib

MAX_SUBMATRIX = 32  # the hafnian path's cap: 2 M cutoff <= 32


def qmat(cov: np.ndarray, hbar: float = 2.0) -> np.ndarray:
    """Husimi Q covariance (a, a-dagger ordering) of an xxpp Wigner covariance."""
    cov = np.asarray(cov, dtype=np.float64)
    n = cov.shape[0] // 2
    x = cov[:n, :n] * (2.0 / hbar)
    p = cov[n:, n:] * (2.0 / hbar)
    xp = cov[:n, n:] * (2.0 / hbar)
    eye = np.eye(n)
    ad_a = (x + p + 1j * (xp - xp.T) - 2.0 * eye) / 4.0   # <a_i^dag a_j>
    a_a = (x - p + 1j * (xp + xp.T)) / 4.0                # <a_i a_j>
    return np.block([[ad_a, a_a.conj()], [a_a, ad_a.conj()]]) + np.eye(2 * n)


def reduced_A(cov: np.ndarray, k: int, hbar: float = 2.0) -> np.ndarray:
    """A = X (I - Q^{-1}) of the state reduced to its first k modes (2k x 2k)."""
    M = cov.shape[0] // 2
    ix = list(range(k)) + list(range(M, M + k))
    Q = qmat(np.asarray(cov)[np.ix_(ix, ix)], hbar)
    X = np.block([[np.zeros((k, k)), np.eye(k)], [np.eye(k), np.zeros((k, k))]])
    return X @ (np.eye(2 * k) - np.linalg.inv(Q))


def _pack(cov: np.ndarray, hbar: float):
    M = cov.shape[0] // 2
    flat, off, tot = [], [], 0
    for k in range(1, M + 1):
        a = np.ascontiguousarray(reduced_A(cov, k, hbar), dtype=np.complex128).reshape(-1)
        off.append(tot)
        flat.append(a)
        tot += a.size
    return np.ascontiguousarray(np.concatenate(flat)), np.array(off, dtype=np.int32), tot


def _check(cov: np.ndarray, cutoff: int) -> int:
    cov = np.asarray(cov)
    if cov.ndim != 2 or cov.shape[0] != cov.shape[1] or cov.shape[0] % 2:
        raise ValueError(f"cov must be a (2M, 2M) xxpp covariance, got shape {cov.shape}")
    M = cov.shape[0] // 2
    if cutoff < 0:
        raise ValueError("cutoff must be non-negative")
    if 2 * M * cutoff > MAX_SUBMATRIX:
        raise ValueError(f"resident sampler: worst-case submatrix 2*M*cutoff={2 * M * cutoff} exceeds the "
                         f"hafnian cap {MAX_SUBMATRIX}; reduce modes or cutoff")
    return M


def sample_resident(cov: np.ndarray, num_samples: int, cutoff: int = 6, hbar: float = 2.0,
                    seed: int | None = None) -> np.ndarray:
    """(num_samples, M) int64 photon counts drawn on the device (see the module text)."""
    M = _check(cov, cutoff)
    if num_samples < 0:
        raise ValueError("num_samples must be non-negative")
    out = np.zeros((num_samples, M), dtype=np.int32)
    if num_samples == 0:
        return out.astype(np.int64)
    ak, off, tot = _pack(np.asarray(cov, dtype=np.float64), hbar)
    invfac = np.array([1.0 / factorial(j) for j in range(cutoff + 1)], dtype=np.float64)
    lib = _lib.load()
    rc = lib.gbs_sampler_sample(_lib.dptr(ak.view(np.float64)), int(tot), _lib.iptr(off), M, int(num_samples),
                                int(cutoff), MAX_SUBMATRIX, _lib.dptr(invfac),
                                0 if seed is None else int(seed) & 0xFFFFFFFFFFFFFFFF, _lib.iptr(out))
    if rc != 0:
        raise RuntimeError(f"gbs_sampler_sample failed (code {rc}): {lib.gbs_sampler_last_error().decode()}")
    return out.astype(np.int64)


def conditional_weights(cov: np.ndarray, k: int, prefixes: np.ndarray, cutoff: int,
                        hbar: float = 2.0) -> np.ndarray:
    """Re haf of mode k's conditional submatrices for the given prefixes (rows of
    photon counts of modes 1..k-1), evaluated on the device: (len(prefixes), cutoff + 1)."""
    M = _check(cov, cutoff)
    pre = np.asarray(prefixes, dtype=np.int32).reshape(len(prefixes), -1)
    state = np.zeros((len(pre), M), dtype=np.int32)
    state[:, :pre.shape[1]] = pre
    ak, off, tot = _pack(np.asarray(cov, dtype=np.float64), hbar)
    w = np.empty((len(pre), cutoff + 1), dtype=np.float64)
    lib = _lib.load()
    rc = lib.gbs_sampler_conditional_weights(_lib.dptr(ak.view(np.float64)), int(tot), _lib.iptr(off), M, int(k),
                                             _lib.iptr(state), len(pre), int(cutoff), _lib.dptr(w))
    if rc != 0:
        raise RuntimeError(f"gbs_sampler_conditional_weights failed (code {rc}): "
                           f"{lib.gbs_sampler_last_error().decode()}")
    return w
