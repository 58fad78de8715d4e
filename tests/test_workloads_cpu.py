"""Synthetic benchmark inputs have the stated shapes and physical properties."""

from __future__ import annotations

import numpy as np

from gbskernels_b200 import workloads as W


def test_haar_is_unitary():
    U = W.haar_unitary(30, np.random.default_rng(0))
    assert np.allclose(U.conj().T @ U, np.eye(30), atol=1e-12)


def test_config1_shapes():
    A = W.haf_real_batch(8, 16, seed=1)
    assert A.shape == (8, 16, 16) and np.isrealobj(A)
    assert np.allclose(A, np.transpose(A, (0, 2, 1)))


def test_config2_submatrices_of_a_unitary():
    P = W.perm_haar_batch(4, 20, seed=2)
    assert P.shape == (4, 20, 20) and P.dtype == np.complex128
    assert np.all(np.abs(P) < 1.0)


def test_config3_mixed_batch():
    funcs, mats = W.mixed_haf_lhaf(200, seed=3)
    dims = {m.shape[0] for m in mats}
    assert dims <= set(range(8, 29, 2)) and len(dims) > 5
    assert set(funcs) == {"haf", "lhaf"}
    for f, m in zip(funcs, mats):
        assert np.allclose(m, m.T)


def test_config4_physical_domain():
    mats = W.tor_click_batch(20, kmin=3, kmax=8, seed=4)
    for O in mats:
        k = O.shape[0] // 2
        assert 3 <= k <= 8 and np.allclose(O, O.T)
        assert np.min(np.linalg.eigvalsh(np.eye(2 * k) - O)) > 0  # I - O_S SPD


def test_serving_stream_mix():
    reqs = W.serving_stream(300, rate=1e4, seed=5)
    t = [r[0] for r in reqs]
    assert all(b >= a for a, b in zip(t, t[1:]))
    precs = [r[2] for r in reqs]
    assert 0.55 < precs.count("fp64") / 300 < 0.85
    assert {r[1] for r in reqs} == {"haf", "lhaf", "tor"}


def test_reference_flop_formulas():
    # haf N=16 real: (n-1) n^2 (n+3) 2^n MACs x 2 = 2.523e6 flops
    assert W.ref_flops("haf", 16, real=True) == 2 * 7 * 64 * 11 * 256
    assert W.ref_flops("perm", 20) == 2 ** 19 * 196
    assert W.ref_flops("tor", 20) == 2 * 2 ** 10 * 91
