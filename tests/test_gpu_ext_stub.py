"""The reference-facing extension module (gbskernels_b200/ext/gbskernels_ext.py) on
the GPU: every entry point the reference package calls, with the reference
extension's argument and return conventions (bindings/gbskernels_ext.cpp:233-390),
checked against the binary128 oracle.  Modelled on the reference's
tests/test_gpu_bindings.py:40-130 (each binding vs an independent truth, the
certified pairs enclosing it, the session equal to the one-shot call)."""

from __future__ import annotations

import importlib
import sys
from pathlib import Path

import numpy as np
import pytest

from conftest import rel_err

pytestmark = pytest.mark.gpu

EXT_DIR = Path(__file__).resolve().parents[1] / "gbskernels_b200" / "ext"
RNG = np.random.default_rng(77)


@pytest.fixture(scope="module")
def ext(gpu):
    sys.path.insert(0, str(EXT_DIR))
    try:
        return importlib.import_module("gbskernels_ext")
    finally:
        sys.path.remove(str(EXT_DIR))


def _sym(B, N):
    X = RNG.standard_normal((B, N, N)) + 1j * RNG.standard_normal((B, N, N))
    return np.ascontiguousarray(0.25 * (X + np.transpose(X, (0, 2, 1))))


def _phys_O(B, n):
    out = []
    for _ in range(B):
        X = RNG.standard_normal((2 * n, 2 * n))
        S = X @ X.T / (2 * n) + np.eye(2 * n)
        O = np.eye(2 * n) - np.linalg.inv(S)
        out.append((O + O.T) / 2)
    return np.stack(out).astype(np.complex128)


def test_ext_flags(ext):
    assert ext.__host_shim__ is False


@pytest.mark.parametrize("name,N", [("haf", 14), ("lhaf", 12), ("perm", 11)])
def test_ext_batched_tiers(ext, orc, name, N):
    stack = _sym(3, N) if name != "perm" else RNG.standard_normal((3, N, N)) + 1j * RNG.standard_normal((3, N, N))
    truth = [getattr(orc, name)(m, "quad") for m in stack]
    v = getattr(ext, name)(stack)
    vd = getattr(ext, f"{name}_dd")(stack)
    vk, absn = getattr(ext, f"{name}_kappa")(stack)
    vc, bc = getattr(ext, f"{name}_certified")(stack)
    assert v.dtype == np.complex128 and v.shape == (3,)
    for i, t in enumerate(truth):
        assert rel_err(v[i], t) < 1e-10
        assert rel_err(vd[i], t) < 1e-15
        assert vk[i] == v[i] and absn[i] >= abs(v[i]) * (1 - 1e-12)
        assert vc[i] == v[i] and abs(vc[i] - t) <= bc[i]
    vdc, bdc = getattr(ext, f"{name}_dd_certified")(stack)
    for i, t in enumerate(truth):
        assert abs(vdc[i] - t) <= bdc[i] * (1 + 1e-12) + 1e-30


def test_ext_tor_paths(ext, orc):
    stack = _phys_O(3, 6)
    truth = [orc.tor(np.real(m), "quad") for m in stack]
    v = ext.tor(stack)
    vd = ext.tor_dd(stack)
    vc, bc = ext.tor_certified(stack)
    vdc, bdc = ext.tor_dd_certified(stack)
    for i, t in enumerate(truth):
        assert rel_err(v[i], t) < 1e-10
        assert rel_err(vd[i], t) < 1e-15
        assert abs(vc[i] - t) <= bc[i] and abs(vdc[i] - t) <= bdc[i] * (1 + 1e-12) + 1e-30
    O = np.real(stack[0])
    assert rel_err(ext.tor_single(O, 3), truth[0]) < 1e-10
    for fn in (ext.tor_single_certified, ext.tor_single_ddcertified):
        val, bnd = fn(O, 3)
        assert abs(val - truth[0]) <= bnd * (1 + 1e-12) + 1e-30
    with pytest.raises(ValueError):
        ext.tor(np.zeros((1, 3, 3), np.complex128))


def test_ext_session_matches_one_shot(ext):
    stack = _sym(4, 10)
    s = ext.Session()
    try:
        assert np.array_equal(s.haf(stack), ext.haf(stack))
        assert np.array_equal(s.lhaf_dd(stack), ext.lhaf_dd(stack))
        r = s.haf_resident(stack)
        import torch
        t = torch.from_dlpack(r)
        assert t.is_cuda and np.array_equal(t.cpu().numpy(), ext.haf(stack))
        before = s.reallocs()
        s.haf(stack)
        assert s.reallocs() == before  # buffers reused
    finally:
        s.close()
    with pytest.raises(RuntimeError):
        s.haf(stack)


def test_ext_sieve_and_errors(ext, orc):
    M = 5
    X = RNG.standard_normal((M, M)) + 1j * RNG.standard_normal((M, M))
    A = 0.3 * (X + X.T)
    g = 0.2 * (RNG.standard_normal(M) + 1j * RNG.standard_normal(M))
    reps = np.array([[1, 0, 2, 1, 0], [2, 1, 1, 0, 2]], np.int32)
    v = ext.lhaf_repeated(A, g, reps)
    vc, bc = ext.lhaf_repeated_certified(A, g, reps)
    for i in range(2):
        t = orc.lhaf_repeated(A, g, reps[i], "quad")
        assert rel_err(v[i], t) < 1e-10 and abs(vc[i] - t) <= bc[i]
    with pytest.raises(RuntimeError):
        ext.haf(_sym(1, 34))  # above the cap: the library refuses, the wrapper raises
