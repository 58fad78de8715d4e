"""The batch walk of the Python binding (`_pointers`: host address and side of
every matrix for gbs_queue_evaluate_ptrs) gives the same result through the C
helper (_hostptr.collect, buffer protocol) and through the Python loop: taken as
they are, C-contiguous complex128 square arrays; converted first, everything else
(transposed and sliced views, real and single-precision arrays, nested lists); the
first matrix that is not square 2-D refused by position with the same message.
No GPU needed."""

from __future__ import annotations

import numpy as np
import pytest


@pytest.fixture(scope="module")
def G():
    import gbskernels_b200
    return gbskernels_b200


def _mix():
    rng = np.random.default_rng(4)
    A = rng.standard_normal((6, 6)) + 1j * rng.standard_normal((6, 6))
    return A, [A, A.T, A.real.copy(), [[1, 2], [3, 4]], A[:4, :4], np.zeros((0, 0), complex),
               A.astype(np.complex64), np.asfortranarray(A), A[::2, ::2], (A + 1).copy()]


def _walk(G, mats, helper, monkeypatch):
    if not helper:
        monkeypatch.setattr(G, "_hostptr", None)
    ptr, dims, keep = G._pointers(mats)
    vals = []  # the bytes each pointer designates, read back through the returned arrays
    pool = {m.ctypes.data: m for m in keep}
    for i, m in enumerate(mats):
        src = pool.get(int(ptr[i]))
        if src is None:
            assert int(ptr[i]) == np.asarray(m).ctypes.data
            src = m
        vals.append(np.asarray(src).copy())
    return dims.copy(), vals, len(keep)


def test_helper_and_python_walk_agree(G, monkeypatch):
    if G._hostptr is None:
        pytest.skip("the C helper is not built")
    A, mats = _mix()
    d1, v1, k1 = _walk(G, mats, True, monkeypatch)
    d2, v2, k2 = _walk(G, mats, False, monkeypatch)
    assert list(d1) == list(d2) == [6, 6, 6, 2, 4, 0, 6, 6, 3, 6]
    assert k1 == k2
    for i, (a, b) in enumerate(zip(v1, v2)):
        assert a.dtype == np.complex128 and np.array_equal(a, b), i
        assert np.array_equal(a, np.asarray(mats[i], dtype=np.complex128)), i
    p, _, _ = G._pointers([A])
    assert int(p[0]) == A.ctypes.data  # taken as it is: no copy


@pytest.mark.parametrize("helper", [True, False])
def test_non_square_refused_by_position(G, monkeypatch, helper):
    if helper and G._hostptr is None:
        pytest.skip("the C helper is not built")
    if not helper:
        monkeypatch.setattr(G, "_hostptr", None)
    A, _ = _mix()
    for bad in (np.zeros((4, 6), complex), np.zeros((2, 2, 2), complex), np.zeros(5, complex)):
        with pytest.raises(ValueError, match=r"matrix #2 must be square 2-D"):
            G._pointers([A, A, bad, np.zeros((3, 5), complex)])
