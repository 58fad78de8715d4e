"""gbskernels_ext -- libgbs_b200.so exposed as the reference's compiled extension.

The reference's Python package (gbskernels/__init__.py:109-136, ``_load_gpu_ext``)
imports a module named ``gbskernels_ext`` from ``$GBSKERNELS_EXT_DIR``.  Pointing
that variable at this directory makes the reference package run on the B200
library unchanged:

    GBSKERNELS_EXT_DIR=<repo>/gbskernels_b200/ext python -c \\
        "import gbskernels; print(gbskernels.haf_batched(stack, backend='gpu'))"

Every function below is one the reference package calls, with the reference
extension's name, argument list and return shape (bindings/gbskernels_ext.cpp:
233-390): a contiguous complex128 ``(B, d, d)`` stack in, a complex128 ``(B,)``
vector out (``(values, aux)`` for the ``*_kappa`` / ``*_certified`` entries), the
torontonian kernels given the mode count ``d / 2``.  Each is one call into the C
ABI (include/gbs_b200.h) with the same symbol the reference binds; errors raise
``RuntimeError`` with the library's message, as the reference's nanobind wrappers
throw ``std::runtime_error``.  ``Session`` mirrors the reference's resident
session (bindings/gbskernels_ext.cpp:172-229, 374-390).
"""

from __future__ import annotations

import ctypes
import os
import sys
from pathlib import Path

import numpy as np

_HERE = Path(__file__).resolve().parent
_LIB_PATH = Path(os.environ.get("GBS_B200_LIB", str(_HERE.parent / "libgbs_b200.so")))
if not _LIB_PATH.exists():
    raise ImportError(f"gbskernels_ext: {_LIB_PATH} is not built (python -m gbskernels_b200.build)")
_lib = ctypes.CDLL(str(_LIB_PATH))
_dp = ctypes.POINTER(ctypes.c_double)
_ip = ctypes.POINTER(ctypes.c_int)
_lib.gbs_last_error.restype = ctypes.c_char_p
_lib.gbs_lhaf_repeated_last_error.restype = ctypes.c_char_p
_lib.gbs_sampler_last_error.restype = ctypes.c_char_p

# compiled for a real device (the reference's gpu_backend_kind() reads this flag)
__host_shim__ = False


def _err(name: str, rc: int, msg_fn=None) -> RuntimeError:
    msg = (msg_fn or _lib.gbs_last_error)()
    return RuntimeError(f"gbskernels: {name} failed (CUDA error {rc}): {msg.decode() if msg else ''}")


def _stack(a) -> np.ndarray:
    s = np.ascontiguousarray(np.asarray(a, dtype=np.complex128))
    if s.ndim != 3 or s.shape[1] != s.shape[2]:
        raise ValueError("gbskernels: each matrix must be square (B, d, d)")
    return s


def _kdim(s: np.ndarray, tor: bool) -> int:
    d = int(s.shape[1])
    if tor and d % 2:
        raise ValueError("torontonian: matrix dimension must be even (2n x 2n)")
    return d // 2 if tor else d


def _eval(name: str, a, tor: bool = False) -> np.ndarray:
    s = _stack(a)
    out = np.empty(s.shape[0], np.complex128)
    if s.shape[0]:
        rc = getattr(_lib, name)(s.ctypes.data_as(_dp), ctypes.c_int(_kdim(s, tor)), ctypes.c_int(s.shape[0]),
                                 out.ctypes.data_as(_dp))
        if rc:
            raise _err(name, rc)
    return out


def _eval_aux(name: str, a, tor: bool = False):
    s = _stack(a)
    out = np.empty(s.shape[0], np.complex128)
    aux = np.empty(s.shape[0], np.float64)
    if s.shape[0]:
        rc = getattr(_lib, name)(s.ctypes.data_as(_dp), ctypes.c_int(_kdim(s, tor)), ctypes.c_int(s.shape[0]),
                                 out.ctypes.data_as(_dp), aux.ctypes.data_as(_dp))
        if rc:
            raise _err(name, rc)
    return out, aux


# ---- batched kernels (bindings/gbskernels_ext.cpp:233-358) --------------------
def perm(a): return _eval("gbs_perm_host", a)
def perm_dd(a): return _eval("gbs_perm_dd_host", a)
def haf(a): return _eval("gbs_haf_host", a)
def haf_dd(a): return _eval("gbs_haf_dd_host", a)
def lhaf(a): return _eval("gbs_lhaf_host", a)
def lhaf_dd(a): return _eval("gbs_lhaf_dd_host", a)
def tor(a): return _eval("gbs_tor_host", a, tor=True)
def tor_dd(a): return _eval("gbs_tor_dd_host", a, tor=True)

def perm_kappa(a): return _eval_aux("gbs_perm_kappa_host", a)
def haf_kappa(a): return _eval_aux("gbs_haf_kappa_host", a)
def lhaf_kappa(a): return _eval_aux("gbs_lhaf_kappa_host", a)
def tor_kappa(a): return _eval_aux("gbs_tor_kappa_host", a, tor=True)

def perm_certified(a): return _eval_aux("gbs_perm_certified_host", a)
def haf_certified(a): return _eval_aux("gbs_haf_certified_host", a)
def lhaf_certified(a): return _eval_aux("gbs_lhaf_certified_host", a)
def tor_certified(a): return _eval_aux("gbs_tor_certified_host", a, tor=True)

def perm_dd_certified(a): return _eval_aux("gbs_perm_dd_certified_host", a)
def haf_dd_certified(a): return _eval_aux("gbs_haf_dd_certified_host", a)
# the certified double-double rungs the reference lacks (its ladder probes them with
# hasattr, so providing them extends its certified tier to lhaf and tor)
def lhaf_dd_certified(a): return _eval_aux("gbs_lhaf_dd_certified_host", a)
def tor_dd_certified(a): return _eval_aux("gbs_tor_dd_certified_host", a, tor=True)


# ---- single-large torontonian (bindings/gbskernels_ext.cpp:257-295) ------------
def _real_O(O) -> np.ndarray:
    M = np.ascontiguousarray(np.asarray(O), dtype=np.float64)
    if M.ndim != 2 or M.shape[0] != M.shape[1] or M.shape[0] % 2 or M.shape[0] > 64:
        raise ValueError("tor_single: O must be (2n, 2n) with 2n <= 64")
    return M


def tor_single(O, g: int) -> float:
    M = _real_O(O)
    v = ctypes.c_double()
    rc = _lib.gbs_tor_recursive_single_host(M.ctypes.data_as(_dp), ctypes.c_int(M.shape[0] // 2), ctypes.c_int(g),
                                            ctypes.byref(v))
    if rc:
        raise _err("gbs_tor_recursive_single_host", rc)
    return v.value


def _tor_single_bound(name: str, O, g: int):
    M = _real_O(O)
    v, e = ctypes.c_double(), ctypes.c_double()
    rc = getattr(_lib, name)(M.ctypes.data_as(_dp), ctypes.c_int(M.shape[0] // 2), ctypes.c_int(g), ctypes.byref(v),
                             ctypes.byref(e))
    if rc:
        raise _err(name, rc)
    return v.value, e.value


def tor_single_certified(O, g: int): return _tor_single_bound("gbs_tor_single_certified_host", O, g)
def tor_single_ddcertified(O, g: int): return _tor_single_bound("gbs_tor_single_ddcertified_host", O, g)


# ---- repeated-row sieve (bindings/gbskernels_ext.cpp:296-346) -------------------
def _sieve_args(A, g, reps):
    A = np.ascontiguousarray(A, dtype=np.complex128)
    g = np.ascontiguousarray(g, dtype=np.complex128)
    r = np.ascontiguousarray(reps, dtype=np.int32)
    if r.ndim == 1:
        r = r[None, :]
    return A, g, r


def lhaf_repeated(A, g, reps) -> np.ndarray:
    A, g, r = _sieve_args(A, g, reps)
    out = np.empty(r.shape[0], np.complex128)
    rc = _lib.gbs_lhaf_repeated_host(A.view(np.float64).ctypes.data_as(_dp), g.view(np.float64).ctypes.data_as(_dp),
                                     ctypes.c_int(A.shape[0]), r.ctypes.data_as(_ip), ctypes.c_int(r.shape[0]),
                                     out.view(np.float64).ctypes.data_as(_dp))
    if rc:
        raise _err("gbs_lhaf_repeated_host", rc, _lib.gbs_lhaf_repeated_last_error)
    return out


def lhaf_repeated_certified(A, g, reps):
    A, g, r = _sieve_args(A, g, reps)
    out = np.empty(r.shape[0], np.complex128)
    bnd = np.empty(r.shape[0], np.float64)
    rc = _lib.gbs_lhaf_repeated_cert_host(A.view(np.float64).ctypes.data_as(_dp),
                                          g.view(np.float64).ctypes.data_as(_dp), ctypes.c_int(A.shape[0]),
                                          r.ctypes.data_as(_ip), ctypes.c_int(r.shape[0]),
                                          out.view(np.float64).ctypes.data_as(_dp), bnd.ctypes.data_as(_dp))
    if rc:
        raise _err("gbs_lhaf_repeated_cert_host", rc, _lib.gbs_lhaf_repeated_last_error)
    return out, bnd


# ---- resident sampler chain (bindings/gbskernels_ext.cpp:361-372) ---------------
def sample_resident(ak, offs, M, num_samples, cutoff, cap, invfac, seed) -> np.ndarray:
    ak = np.ascontiguousarray(ak, dtype=np.complex128)
    offs = np.ascontiguousarray(offs, dtype=np.int32)
    invfac = np.ascontiguousarray(invfac, dtype=np.float64)
    out = np.zeros((int(num_samples), int(M)), np.int32)
    rc = _lib.gbs_sampler_sample(ak.view(np.float64).ctypes.data_as(_dp), ctypes.c_int(ak.size),
                                 offs.ctypes.data_as(_ip), ctypes.c_int(M), ctypes.c_int(num_samples),
                                 ctypes.c_int(cutoff), ctypes.c_int(cap), invfac.ctypes.data_as(_dp),
                                 ctypes.c_ulonglong(seed), out.ctypes.data_as(_ip))
    if rc:
        raise _err("gbs_sampler_sample", rc, _lib.gbs_sampler_last_error)
    return out


# ---- resident session (bindings/gbskernels_ext.cpp:172-229, 374-390) ------------
class _DeviceResult:
    """(B,) complex128 results left on the device (DLPack export, zero copy), freed
    with gbs_dev_free when the last consumer lets go."""

    def __init__(self, ptr, n: int):
        if str(_HERE.parents[1]) not in sys.path:
            sys.path.insert(0, str(_HERE.parents[1]))
        from gbskernels_b200 import _ResidentResult
        self._r = _ResidentResult(ptr, n)

    def __dlpack__(self, stream=None):
        return self._r.__dlpack__(stream)

    def __dlpack_device__(self):
        return self._r.__dlpack_device__()

    @property
    def __cuda_array_interface__(self):
        return self._r.__cuda_array_interface__

    def __len__(self):
        return len(self._r)

    def get(self) -> np.ndarray:
        """Copy to the host (the CuPy name)."""
        return self._r.numpy()


class Session:
    """One device-resident session: buffers reused across calls, synchronous
    evaluate (func 0 perm, 1 haf, 2 lhaf, 3 tor; prec 0 fp64, 1 dd)."""

    def __init__(self):
        self._s = ctypes.c_void_p()
        rc = _lib.gbs_session_open(ctypes.byref(self._s))
        if rc:
            raise _err("gbs_session_open", rc)

    def _call(self, func: int, prec: int, a, tor: bool) -> np.ndarray:
        if not self._s:
            raise RuntimeError("gbskernels: session is closed")
        s = _stack(a)
        _kdim(s, tor)  # validates the even side of a torontonian
        d = int(s.shape[1])  # sessions take the matrix side
        out = np.empty(s.shape[0], np.complex128)
        rc = _lib.gbs_session_evaluate(self._s, ctypes.c_int(func), ctypes.c_int(prec), s.ctypes.data_as(_dp),
                                       ctypes.c_int(d), ctypes.c_int(s.shape[0]), out.ctypes.data_as(_dp))
        if rc:
            raise _err("gbs_session_evaluate", rc)
        return out

    def _call_resident(self, func: int, a, tor: bool) -> _DeviceResult:
        if not self._s:
            raise RuntimeError("gbskernels: session is closed")
        s = _stack(a)
        _kdim(s, tor)
        d = int(s.shape[1])
        ptr = _dp()
        rc = _lib.gbs_session_evaluate_resident(self._s, ctypes.c_int(func), ctypes.c_int(0), s.ctypes.data_as(_dp),
                                                ctypes.c_int(d), ctypes.c_int(s.shape[0]), ctypes.byref(ptr))
        if rc:
            raise _err("gbs_session_evaluate_resident", rc)
        return _DeviceResult(ptr, s.shape[0])

    def perm(self, a): return self._call(0, 0, a, False)
    def perm_dd(self, a): return self._call(0, 1, a, False)
    def haf(self, a): return self._call(1, 0, a, False)
    def haf_dd(self, a): return self._call(1, 1, a, False)
    def lhaf(self, a): return self._call(2, 0, a, False)
    def lhaf_dd(self, a): return self._call(2, 1, a, False)
    def tor(self, a): return self._call(3, 0, a, True)
    def tor_dd(self, a): return self._call(3, 1, a, True)
    def perm_resident(self, a): return self._call_resident(0, a, False)
    def haf_resident(self, a): return self._call_resident(1, a, False)
    def lhaf_resident(self, a): return self._call_resident(2, a, False)
    def tor_resident(self, a): return self._call_resident(3, a, True)

    def close(self) -> None:
        if self._s:
            _lib.gbs_session_close(self._s)
            self._s = ctypes.c_void_p()

    def reallocs(self) -> int:
        if not self._s:
            return 0
        _lib.gbs_session_reallocs.restype = ctypes.c_size_t
        return int(_lib.gbs_session_reallocs(self._s))

    def __del__(self):  # pragma: no cover
        try:
            self.close()
        except Exception:
            pass
