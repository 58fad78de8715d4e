"""gbs_haf_noalloc: the hafnian entry point for callers that cannot allocate device
memory at evaluation time (their memory belongs to another allocator, or an
allocation would stall a latency-critical loop).  It takes device pointers for the
input matrices and the output, and keeps all scratch in a fixed 4 MiB array inside
the library.  Checked through the C ABI against gbs_haf_host on the same inputs:
two calls in a row (the second smaller, over the first call's leftovers), the
trivial sides (N = 0 and odd N), both limits hit exactly, and refusals of
oversize requests whose buffers are sized for the whole request (a wrongly
accepted call then fails the assertion without touching foreign memory)."""

from __future__ import annotations

import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(autouse=True)
def _untuned(lib):
    # the default split (7) fixes the item counts these cases are sized for
    from gbskernels_b200 import autotune
    autotune.clear()
    yield


def _sym(rng, B, N):
    X = rng.standard_normal((B, N, N)) + 1j * rng.standard_normal((B, N, N))
    return np.ascontiguousarray(0.5 * (X + np.transpose(X, (0, 2, 1))) / 2)


def _haf_host(lib, stack):
    out = np.empty(stack.shape[0], dtype=np.complex128)
    dp = ctypes.POINTER(ctypes.c_double)
    rc = lib.gbs_haf_host(stack.ctypes.data_as(dp), stack.shape[1], stack.shape[0], out.ctypes.data_as(dp))
    assert rc == 0
    return out


def _fn(lib):
    fn = lib.gbs_haf_noalloc
    fn.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p]
    fn.restype = ctypes.c_int
    return fn


def _haf_noalloc(lib, stack):
    import torch
    B, N = stack.shape[0], stack.shape[1]
    d_in = torch.from_numpy(stack.view(np.float64).reshape(-1).copy()).cuda()
    # the output starts as NaN so that an element the call does not write is caught
    d_out = torch.full((2 * B,), float("nan"), dtype=torch.float64, device="cuda")
    s = torch.cuda.current_stream()
    rc = _fn(lib)(d_in.data_ptr(), N, B, d_out.data_ptr(), s.cuda_stream)
    if rc != 0:
        lib.gbs_haf_noalloc_last_error.restype = ctypes.c_char_p
        pytest.fail(f"gbs_haf_noalloc returned {rc}: {lib.gbs_haf_noalloc_last_error().decode()}")
    torch.cuda.synchronize()
    return d_out.cpu().numpy().view(np.complex128)


def test_noalloc_matches_host_entry_point_twice(lib):
    rng = np.random.default_rng(2024)
    first = _sym(rng, 64, 22)
    second = _sym(rng, 9, 14)
    for stack in (first, second):
        got = _haf_noalloc(lib, stack)
        ref = _haf_host(lib, stack)
        assert np.allclose(got, ref, rtol=1e-10, atol=0.0)
        assert np.array_equal(got, ref)


def test_noalloc_real_input_agrees_to_rounding(lib):
    # a real input runs the real power loop through gbs_haf_host and the complex one
    # here: equal to rounding, not bit for bit
    rng = np.random.default_rng(31)
    for N in (12, 20):
        stack = np.ascontiguousarray(_sym(rng, 16, N).real.astype(np.complex128))
        got = _haf_noalloc(lib, stack)
        ref = _haf_host(lib, stack)
        assert np.all(np.isfinite(got))
        assert np.allclose(got, ref, rtol=1e-10, atol=0.0), (N, np.max(np.abs(got - ref) / np.abs(ref)))


def test_noalloc_trivial_sides(lib):
    rng = np.random.default_rng(7)
    # N = 0: haf = 1; odd N: haf = 0 -- written by the library, not left over
    for N, want in ((0, 1.0), (5, 0.0), (13, 0.0)):
        stack = np.zeros((33, N, N), np.complex128) if N == 0 else _sym(rng, 33, N)
        got = _haf_noalloc(lib, stack)
        assert np.array_equal(got, np.full(33, want, np.complex128))
        assert np.array_equal(got, _haf_host(lib, stack))
    # and a real evaluation right after, over those calls' leftovers
    stack = _sym(rng, 17, 12)
    assert np.array_equal(_haf_noalloc(lib, stack), _haf_host(lib, stack))


def test_noalloc_exact_limits(lib):
    rng = np.random.default_rng(11)
    # 12288 instances x 2^(9-7) items = 49152 work items: the item limit exactly
    stack = _sym(rng, 12288, 18)
    assert np.array_equal(_haf_noalloc(lib, stack), _haf_host(lib, stack))
    # 16384 instances of N = 8 (one item each): the instance limit exactly
    stack = _sym(rng, 16384, 8)
    assert np.array_equal(_haf_noalloc(lib, stack), _haf_host(lib, stack))


def test_noalloc_rejects_oversize(lib):
    import torch
    fn = _fn(lib)

    def refused(B, N):
        d_in = torch.zeros(max(1, 2 * B * N * N), dtype=torch.float64, device="cuda")
        d_out = torch.zeros(max(2, 2 * B), dtype=torch.float64, device="cuda")
        rc = fn(d_in.data_ptr(), N, B, d_out.data_ptr(), None)
        torch.cuda.synchronize()
        return rc != 0

    # 100 x 2^(16-7) = 51200 > 49152 items; one item past the limit; one instance past it
    assert refused(100, 32)
    assert refused(12289, 18)
    assert refused(16385, 8)
    assert refused(1, 34)  # N above 32
