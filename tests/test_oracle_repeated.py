"""Pin of the oracle's finite-difference sieve (repeated-row loop hafnian) against
the reference's golden fixtures: its binary64 sieve (cpu_ref.lhaf_repeated) and the
40-digit mpmath loop hafnian of the expanded matrix (tests/golden/golden_repeated.npz,
generator tests/golden/make_golden_repeated.py).  CPU only."""

from __future__ import annotations

from pathlib import Path

import numpy as np
import pytest

from conftest import rel_err

G = Path(__file__).resolve().parent / "golden" / "golden_repeated.npz"


@pytest.fixture(scope="module")
def rep():
    return dict(np.load(G))


def _case(rep, i):
    M = int(rep["M"][i])
    mp = rep["mp"][i]
    truth = complex(mp[0] + mp[1], mp[2] + mp[3])
    return rep["A"][i][:M, :M], rep["gamma"][i][:M], rep["reps"][i][:M], truth


def test_oracle_sieve_matches_mpmath_of_the_expansion(orc, rep):
    for i in range(len(rep["M"])):
        A, g, r, truth = _case(rep, i)
        q = orc.lhaf_repeated(A, g, r, "quad")
        assert rel_err(q, truth) < 1e-14 or abs(q - truth) < 1e-14, (i, q, truth)


def test_oracle_sieve_binary64_tracks_the_reference_sieve(orc, rep):
    for i in range(len(rep["M"])):
        A, g, r, truth = _case(rep, i)
        v = orc.lhaf_repeated(A, g, r, "fp64")
        ref = complex(rep["cpu_sieve"][i])
        assert abs(v - ref) <= 1e-12 * max(abs(truth), 1.0), (i, v, ref)


def test_oracle_sieve_equals_the_expanded_power_trace(orc, rep):
    # the sieve and the power trace of the expansion are two algorithms for one value
    for i in range(0, len(rep["M"]), 3):
        A, g, r, truth = _case(rep, i)
        idx = np.repeat(np.arange(len(r)), r)
        E = A[np.ix_(idx, idx)].copy()
        np.fill_diagonal(E, g[idx])
        assert rel_err(orc.lhaf(E, "quad"), orc.lhaf_repeated(A, g, r, "quad")) < 1e-25 or \
            abs(orc.lhaf(E, "quad") - orc.lhaf_repeated(A, g, r, "quad")) < 1e-25
