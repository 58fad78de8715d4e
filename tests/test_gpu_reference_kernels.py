"""The reference's own GPU path as a comparison arm.

oracle/Makefile (target ref-gpu) compiles the reference's core/*.cu unchanged with
nvcc for sm_100a into oracle/_ref/libgbsref_gpu.so (test infrastructure, never the
product; skipped where it was not built).  Its batched hafnian and loop hafnian are
one thread per instance with per-thread buffers capped at N = 20
(core/hafnian.cu:116-161, core/loop_hafnian.cu:113-140), and its plain per-size
path is one synchronous session call per (function, size) bucket: stage, H2D,
launch, D2H, stream sync (core/host_api.cu:537-590), driven bucket by bucket from
the Python workspace with a host scatter (gbskernels/__init__.py:813-852).

  * parity: on the config-3 mix restricted to the reference's cap (N = 8..20), the
    reference kernels' values agree with this library's within
    1e-10 |v| + 32 N u sum|term| (the two walks round differently);
  * speed: the persistent mixed-size queue (Workspace.evaluate, numpy in, numpy
    out) against that per-size path on the same instances, end to end on both
    sides; the persistent queue must be at least 3x faster.  The measured times
    are printed as one JSON line (run with -s to see it).
"""

from __future__ import annotations

import ctypes
import json
import time
from pathlib import Path

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

REF_GPU = Path(__file__).resolve().parents[1] / "oracle" / "_ref" / "libgbsref_gpu.so"
U = 2.0 ** -53
FCODE = {"perm": 0, "haf": 1, "lhaf": 2, "tor": 3}


@pytest.fixture(scope="module")
def ref():
    if not REF_GPU.exists():
        pytest.skip("the reference's GPU build (oracle/_ref/libgbsref_gpu.so) is not present")
    lib = ctypes.CDLL(str(REF_GPU))  # RTLD_LOCAL: its gbs_* names stay in this handle
    vp, dp = ctypes.c_void_p, ctypes.POINTER(ctypes.c_double)
    lib.gbs_session_open.argtypes = [ctypes.POINTER(vp)]
    lib.gbs_session_open.restype = ctypes.c_int
    lib.gbs_session_evaluate.argtypes = [vp, ctypes.c_int, ctypes.c_int, dp, ctypes.c_int, ctypes.c_int, dp]
    lib.gbs_session_evaluate.restype = ctypes.c_int
    lib.gbs_session_close.argtypes = [vp]
    lib.gbs_session_close.restype = ctypes.c_int
    return lib


def _ref_per_size(ref, sess, funcs, mats):
    """The reference's plain per-size path: buckets in first-seen order, one
    synchronous session call each, scatter back to input order."""
    dp = ctypes.POINTER(ctypes.c_double)
    buckets: dict = {}
    for i, (f, m) in enumerate(zip(funcs, mats)):
        buckets.setdefault((f, m.shape[0]), []).append(i)
    out = np.empty(len(mats), np.complex128)
    for (f, d), idx in buckets.items():
        stack = np.ascontiguousarray(np.stack([mats[i] for i in idx]))
        res = np.empty(len(idx), np.complex128)
        rc = ref.gbs_session_evaluate(sess, FCODE[f], 0, stack.view(np.float64).ctypes.data_as(dp), d, len(idx),
                                      res.view(np.float64).ctypes.data_as(dp))
        assert rc == 0, (f, d, rc)
        out[idx] = res
    return out


def _mix_within_cap(B, seed):
    from gbskernels_b200 import workloads
    funcs, mats = workloads.mixed_haf_lhaf(B, seed=seed)
    keep = [i for i, m in enumerate(mats) if m.shape[0] <= 20]
    return [funcs[i] for i in keep], [mats[i] for i in keep]


def test_reference_gpu_kernels_agree(gpu, ref):
    funcs, mats = _mix_within_cap(512, seed=11)
    sess = ctypes.c_void_p()
    assert ref.gbs_session_open(ctypes.byref(sess)) == 0
    try:
        r = _ref_per_size(ref, sess, funcs, mats)
    finally:
        ref.gbs_session_close(sess)
    with gpu.Workspace() as ws:
        v, absn, st = ws.evaluate_full(funcs, mats, ["kappa"] * len(mats))
    assert (st == 0).all()
    for i, m in enumerate(mats):
        tol = 1e-10 * abs(v[i]) + 32 * m.shape[0] * U * absn[i]
        assert abs(r[i] - v[i]) <= tol, (funcs[i], m.shape[0], r[i], v[i], absn[i] / abs(v[i]))


def test_persistent_queue_against_reference_per_size_path(gpu, ref):
    funcs, mats = _mix_within_cap(4096, seed=12)
    B = len(mats)
    precs = ["fp64"] * B
    sess = ctypes.c_void_p()
    assert ref.gbs_session_open(ctypes.byref(sess)) == 0
    try:
        with gpu.Workspace() as ws:
            ours = ws.evaluate(funcs, mats, precs)  # warm-up (plan, buffers, graphs)
            theirs = _ref_per_size(ref, sess, funcs, mats)
            t_ours, t_ref = [], []
            for _ in range(3):
                t0 = time.perf_counter()
                o = ws.evaluate(funcs, mats, precs)
                t_ours.append(time.perf_counter() - t0)
            for _ in range(2):
                t0 = time.perf_counter()
                rr = _ref_per_size(ref, sess, funcs, mats)
                t_ref.append(time.perf_counter() - t0)
    finally:
        ref.gbs_session_close(sess)
    assert np.array_equal(o, ours)
    assert np.array_equal(rr, theirs)
    t_o, t_r = float(np.median(t_ours)), float(np.median(t_ref))
    sizes = sorted({m.shape[0] for m in mats})
    print(json.dumps({"instances": B, "sizes": sizes, "persistent_ms": 1e3 * t_o, "reference_per_size_ms": 1e3 * t_r,
                      "speedup": t_r / t_o, "buckets": len({(f, m.shape[0]) for f, m in zip(funcs, mats)})}))
    assert t_r / t_o >= 3.0, (t_o, t_r)
