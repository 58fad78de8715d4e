"""gbs_haf_noalloc: the hafnian entry point for callers that cannot allocate device
memory at evaluation time (their memory belongs to another allocator, or an
allocation would stall a latency-critical loop).  It takes device pointers for the
input matrices and the output, and keeps all scratch in a fixed 4 MiB array inside
the library.  Checked through the C ABI against gbs_haf_host on the same inputs,
on two calls in a row (the second smaller, over the first call's leftovers)."""

from __future__ import annotations

import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _haf_host(lib, stack):
    out = np.empty(stack.shape[0], dtype=np.complex128)
    dp = ctypes.POINTER(ctypes.c_double)
    rc = lib.gbs_haf_host(stack.ctypes.data_as(dp), stack.shape[1], stack.shape[0], out.ctypes.data_as(dp))
    assert rc == 0
    return out


def _haf_noalloc(lib, stack):
    import torch
    fn = lib.gbs_haf_noalloc
    fn.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p]
    fn.restype = ctypes.c_int
    d_in = torch.from_numpy(stack.view(np.float64).copy()).cuda()
    d_out = torch.empty(2 * stack.shape[0], dtype=torch.float64, device="cuda")
    s = torch.cuda.current_stream()
    rc = fn(d_in.data_ptr(), stack.shape[1], stack.shape[0], d_out.data_ptr(), s.cuda_stream)
    if rc != 0:
        lib.gbs_haf_noalloc_last_error.restype = ctypes.c_char_p
        pytest.fail(f"gbs_haf_noalloc returned {rc}: {lib.gbs_haf_noalloc_last_error().decode()}")
    torch.cuda.synchronize()
    return d_out.cpu().numpy().view(np.complex128)


def test_noalloc_matches_host_entry_point_twice(lib):
    rng = np.random.default_rng(2024)

    def batch(B, N):
        X = rng.standard_normal((B, N, N)) + 1j * rng.standard_normal((B, N, N))
        return np.ascontiguousarray(0.5 * (X + np.transpose(X, (0, 2, 1))) / 2)

    first = batch(64, 22)
    second = batch(9, 14)
    for stack in (first, second):
        got = _haf_noalloc(lib, stack)
        ref = _haf_host(lib, stack)
        assert np.allclose(got, ref, rtol=1e-10, atol=0.0)
        assert np.array_equal(got, ref)


def test_noalloc_rejects_oversize(lib):
    import torch
    fn = lib.gbs_haf_noalloc
    fn.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p]
    fn.restype = ctypes.c_int
    d = torch.zeros(2, dtype=torch.float64, device="cuda")
    # 2^(16-7) items per instance x 100 instances = 51200 > 49152: refused before any launch
    assert fn(d.data_ptr(), 32, 100, d.data_ptr(), None) != 0
    assert fn(d.data_ptr(), 34, 1, d.data_ptr(), None) != 0
