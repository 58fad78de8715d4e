"""CPU oracle for the batched perm / haf / lhaf / tor path -- TEST INFRASTRUCTURE.

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline / reference
arm may import this package, and only as the checker or as the timed CPU baseline.
The product path (``gbskernels_b200``) never imports it and has no CPU fallback.

Two checkers live here:

* ``liboracle.so`` -- this repository's restatement of the reference algorithms
  (``gbs_oracle.cpp``), in binary64 and in binary128 (``__float128``).  Citations to
  the reference's files are in that source.
* ``_ref/libgbsref.so`` -- the reference's OWN kernel sources (core/*.cu) compiled
  unchanged as host C++ through the reference's pre-flight shim
  (core/preflight/cuda/*.h) by ``oracle/Makefile``.  Its ``gbs_*_host`` entry points
  (core/host_api.cu:150-268) run the reference kernels on the host with a serial grid
  emulation.  Present when the reference tree was available at build time.

The pin of both against golden vectors lives in ``tests/test_oracle_golden.py``.
"""

from __future__ import annotations

import ctypes
import os
from pathlib import Path

import numpy as np

_HERE = Path(__file__).resolve().parent
_ORC = None
_REF = None

_dp = ctypes.POINTER(ctypes.c_double)


def _load_oracle():
    global _ORC
    if _ORC is None:
        path = _HERE / "liboracle.so"
        if not path.exists():
            raise RuntimeError(f"oracle not built: run `make -C {_HERE}`")
        lib = ctypes.CDLL(str(path))
        for name in ("orc_perm", "orc_haf", "orc_lhaf", "orc_tor_real", "orc_tor_complex"):
            fn = getattr(lib, name)
            fn.argtypes = [_dp, ctypes.c_int, ctypes.c_int, _dp, _dp]
            fn.restype = ctypes.c_int
        _ORC = lib
    return _ORC


def ref_available() -> bool:
    return (_HERE / "_ref" / "libgbsref.so").exists()


def _load_ref():
    global _REF
    if _REF is None:
        path = _HERE / "_ref" / "libgbsref.so"
        if not path.exists():
            raise RuntimeError("reference shim library not built (oracle/_ref/libgbsref.so)")
        _REF = ctypes.CDLL(str(path))
    return _REF


def _call(name: str, A, dim_arg: int, prec: int, real: bool = False):
    lib = _load_oracle()
    if real:
        a = np.ascontiguousarray(np.real(np.asarray(A)), dtype=np.float64)
    else:
        a = np.ascontiguousarray(np.asarray(A, dtype=np.complex128))
    out = np.zeros(4, dtype=np.float64)
    absn = np.zeros(1, dtype=np.float64)
    rc = getattr(lib, name)(a.ctypes.data_as(_dp), dim_arg, prec,
                            out.ctypes.data_as(_dp), absn.ctypes.data_as(_dp))
    if rc != 0:
        raise ValueError(f"{name}: size out of the oracle's range")
    return out, float(absn[0])


def _value(out: np.ndarray, hilo: bool):
    if hilo:
        return (out[0], out[1], out[2], out[3])
    return complex(out[0] + out[1], out[2] + out[3])


def perm(A, prec: str = "fp64", hilo: bool = False, with_absnorm: bool = False):
    """Permanent (Glynn Gray-code walk). prec 'fp64' or 'quad' (binary128)."""
    A = np.asarray(A)
    out, absn = _call("orc_perm", A, A.shape[0], 0 if prec == "fp64" else 1)
    v = _value(out, hilo)
    return (v, absn) if with_absnorm else v


def haf(A, prec: str = "fp64", hilo: bool = False, with_absnorm: bool = False):
    """Hafnian (power trace, diagonal ignored)."""
    A = np.asarray(A)
    out, absn = _call("orc_haf", A, A.shape[0], 0 if prec == "fp64" else 1)
    v = _value(out, hilo)
    return (v, absn) if with_absnorm else v


def lhaf(A, prec: str = "fp64", hilo: bool = False, with_absnorm: bool = False):
    """Loop hafnian (power trace with the loop term; odd N augmented)."""
    A = np.asarray(A)
    out, absn = _call("orc_lhaf", A, A.shape[0], 0 if prec == "fp64" else 1)
    v = _value(out, hilo)
    return (v, absn) if with_absnorm else v


def tor(O, prec: str = "fp64", hilo: bool = False, with_absnorm: bool = False):
    """Torontonian: recursive prefix Cholesky for real O (NaN off-domain), otherwise
    the per-subset complex LU determinant."""
    O = np.asarray(O)
    n = O.shape[0] // 2
    p = 0 if prec == "fp64" else 1
    if not np.iscomplexobj(O) or not np.any(np.imag(O) != 0):
        out, absn = _call("orc_tor_real", O, n, p, real=True)
        if np.isfinite(out[0]):
            v = _value(out, hilo)
            return (v, absn) if with_absnorm else v
    out, absn = _call("orc_tor_complex", O, n, p)
    v = _value(out, hilo)
    return (v, absn) if with_absnorm else v


def lhaf_repeated(A, gamma, reps, prec: str = "fp64"):
    """Loop hafnian of A with row/col i repeated reps[i] times (loop weight gamma[i]
    on every copy), by the finite-difference sieve (cpu_ref/repeated.py:64-122)."""
    lib = _load_oracle()
    A = np.ascontiguousarray(A, dtype=np.complex128)
    M = A.shape[0]
    g = np.zeros(M, np.complex128) if gamma is None else np.ascontiguousarray(gamma, dtype=np.complex128)
    r = np.ascontiguousarray(reps, dtype=np.int32)
    out = np.zeros(4)
    fn = lib.orc_lhaf_repeated
    fn.argtypes = [_dp, _dp, ctypes.POINTER(ctypes.c_int), ctypes.c_int, ctypes.c_int, _dp]
    fn.restype = ctypes.c_int
    rc = fn(A.view(np.float64).ctypes.data_as(_dp), g.view(np.float64).ctypes.data_as(_dp),
            r.ctypes.data_as(ctypes.POINTER(ctypes.c_int)), M, 0 if prec == "fp64" else 1,
            out.ctypes.data_as(_dp))
    if rc:
        raise ValueError("orc_lhaf_repeated: bad arguments")
    return _value(out, False)


def tor_complex(O, prec: str = "fp64"):
    O = np.asarray(O)
    out, _ = _call("orc_tor_complex", O, O.shape[0] // 2, 0 if prec == "fp64" else 1)
    return _value(out, False)


# --- the reference's own kernels (host-shim build) ---------------------------

_REF_FNS = {
    ("perm", "fp64"): "gbs_perm_host", ("perm", "dd"): "gbs_perm_dd_host",
    ("haf", "fp64"): "gbs_haf_host", ("haf", "dd"): "gbs_haf_dd_host",
    ("lhaf", "fp64"): "gbs_lhaf_host", ("lhaf", "dd"): "gbs_lhaf_dd_host",
    ("tor", "fp64"): "gbs_tor_host", ("tor", "dd"): "gbs_tor_dd_host",
}
_REF_AUX_FNS = {
    ("perm", "kappa"): "gbs_perm_kappa_host", ("haf", "kappa"): "gbs_haf_kappa_host",
    ("lhaf", "kappa"): "gbs_lhaf_kappa_host", ("tor", "kappa"): "gbs_tor_kappa_host",
    ("perm", "certified"): "gbs_perm_certified_host", ("haf", "certified"): "gbs_haf_certified_host",
    ("lhaf", "certified"): "gbs_lhaf_certified_host", ("tor", "certified"): "gbs_tor_certified_host",
}


def ref_batched(func: str, stack, tier: str = "fp64"):
    """Run the reference's own host entry point (core/host_api.cu:150-268) on a
    uniform (B, d, d) complex128 stack.  Returns values, or (values, aux) for the
    'kappa' / 'certified' tiers."""
    lib = _load_ref()
    stack = np.ascontiguousarray(np.asarray(stack, dtype=np.complex128))
    B, d = stack.shape[0], stack.shape[1]
    dim = d // 2 if func == "tor" else d
    out = np.zeros(B, dtype=np.complex128)
    if tier in ("fp64", "dd"):
        fn = getattr(lib, _REF_FNS[(func, tier)])
        rc = fn(ctypes.c_void_p(stack.ctypes.data), ctypes.c_int(dim), ctypes.c_int(B),
                ctypes.c_void_p(out.ctypes.data))
        if rc != 0:
            raise RuntimeError(f"reference {func}/{tier} returned {rc}")
        return out
    aux = np.zeros(B, dtype=np.float64)
    fn = getattr(lib, _REF_AUX_FNS[(func, tier)])
    rc = fn(ctypes.c_void_p(stack.ctypes.data), ctypes.c_int(dim), ctypes.c_int(B),
            ctypes.c_void_p(out.ctypes.data), ctypes.c_void_p(aux.ctypes.data))
    if rc != 0:
        raise RuntimeError(f"reference {func}/{tier} returned {rc}")
    return out, aux


def ref_tor_single_ddcertified(O, groups: int = 0):
    """The reference's certified double-double single-large recursive torontonian
    (core/tor_recursive.cu:523-678 via core/host_api.cu gbs_tor_single_ddcertified_host):
    a rigorous enclosure for real O, used as the truth for large mode counts."""
    lib = _load_ref()
    M = np.ascontiguousarray(np.real(np.asarray(O)), dtype=np.float64)
    n = M.shape[0] // 2
    v = ctypes.c_double(0.0)
    e = ctypes.c_double(0.0)
    rc = lib.gbs_tor_single_ddcertified_host(M.ctypes.data_as(_dp), ctypes.c_int(n),
                                             ctypes.c_int(groups), ctypes.byref(v), ctypes.byref(e))
    if rc != 0:
        raise RuntimeError(f"reference tor_single_ddcertified returned {rc}")
    return v.value, e.value


def cores() -> int:
    return len(os.sched_getaffinity(0))
