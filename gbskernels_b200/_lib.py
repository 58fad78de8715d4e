"""ctypes binding to libgbs_b200.so (the C ABI declared in include/gbs_b200.h).

The library is loaded from this package directory (built in-tree by
``gbskernels_b200.build``).  There is no fallback: if the library is missing or
cannot load, every GPU entry point raises ``RuntimeError``.
"""

from __future__ import annotations

import ctypes
import os
from pathlib import Path

import numpy as np

_HERE = Path(__file__).resolve().parent
LIB_PATH = _HERE / "libgbs_b200.so"

_dp = ctypes.POINTER(ctypes.c_double)
_ip = ctypes.POINTER(ctypes.c_int)
_llp = ctypes.POINTER(ctypes.c_longlong)
_vp = ctypes.c_void_p

# name -> (argtypes, restype)
SIGNATURES: dict[str, tuple[list, object]] = {
    "gbs_version": ([], ctypes.c_int),
    "gbs_last_error": ([], ctypes.c_char_p),
    # one-shot uniform batches: (mats, dim, batch, out)
    **{f"gbs_{f}_host": ([_dp, ctypes.c_int, ctypes.c_int, _dp], ctypes.c_int)
       for f in ("perm", "perm_dd", "haf", "haf_dd", "lhaf", "lhaf_dd", "tor", "tor_dd")},
    # value + per-element double (sum|term| or certified bound)
    **{f"gbs_{f}_{k}_host": ([_dp, ctypes.c_int, ctypes.c_int, _dp, _dp], ctypes.c_int)
       for f in ("perm", "haf", "lhaf", "tor") for k in ("kappa", "certified")},
    # value + certified double-double bound
    **{f"gbs_{f}_dd_certified_host": ([_dp, ctypes.c_int, ctypes.c_int, _dp, _dp], ctypes.c_int)
       for f in ("perm", "haf", "lhaf", "tor")},
    "gbs_auto_host": ([ctypes.c_int, _dp, ctypes.c_int, ctypes.c_int, ctypes.c_double, _dp, _dp, _ip],
                      ctypes.c_int),
    "gbs_certified_ladder_host": ([ctypes.c_int, _dp, ctypes.c_int, ctypes.c_int, ctypes.c_double, _dp, _dp, _ip],
                                  ctypes.c_int),
    "gbs_queue_evaluate_auto": ([_vp, ctypes.c_int, _ip, _ip, _llp, _dp, ctypes.c_double, _dp, _dp, _ip, _ip],
                                ctypes.c_int),
    # single-large torontonian
    "gbs_tor_recursive_single_host": ([_dp, ctypes.c_int, ctypes.c_int, _dp], ctypes.c_int),
    "gbs_tor_single_certified_host": ([_dp, ctypes.c_int, ctypes.c_int, _dp, _dp], ctypes.c_int),
    "gbs_tor_single_ddcertified_host": ([_dp, ctypes.c_int, ctypes.c_int, _dp, _dp], ctypes.c_int),
    # sessions
    "gbs_session_open": ([ctypes.POINTER(_vp)], ctypes.c_int),
    "gbs_session_close": ([_vp], ctypes.c_int),
    "gbs_session_reallocs": ([_vp], ctypes.c_size_t),
    "gbs_session_evaluate": ([_vp, ctypes.c_int, ctypes.c_int, _dp, ctypes.c_int, ctypes.c_int, _dp],
                             ctypes.c_int),
    "gbs_session_evaluate_resident": ([_vp, ctypes.c_int, ctypes.c_int, _dp, ctypes.c_int, ctypes.c_int,
                                       ctypes.POINTER(_dp)], ctypes.c_int),
    "gbs_session_evaluate_resident_tier": ([_vp, ctypes.c_int, ctypes.c_int, _dp, ctypes.c_int, ctypes.c_int,
                                            ctypes.POINTER(_dp)], ctypes.c_int),
    "gbs_queue_evaluate_resident": ([_vp, ctypes.c_int, _ip, _ip, _ip, _llp, _dp, ctypes.c_int,
                                     ctypes.POINTER(_dp)], ctypes.c_int),
    "gbs_dev_copy_to_host": ([_vp, _vp, ctypes.c_size_t], ctypes.c_int),
    "gbs_dev_device": ([_vp, _ip], ctypes.c_int),
    "gbs_dev_to_host": ([_dp, _dp, ctypes.c_int], ctypes.c_int),
    "gbs_dev_free": ([_dp], ctypes.c_int),
    "gbs_queue_evaluate": ([_vp, ctypes.c_int, _ip, _ip, _ip, _llp, _dp, ctypes.c_int, _dp, _dp, _ip],
                           ctypes.c_int),
    "gbs_queue_evaluate_ptrs": ([_vp, ctypes.c_int, _ip, _ip, _ip, _vp, ctypes.c_int, _dp, _dp, _ip],
                                ctypes.c_int),
    "gbs_session_last_stats": ([_vp, _dp, _ip, _llp], ctypes.c_int),
    "gbs_queue_prepare": ([_vp, ctypes.c_int, _ip, _ip, _ip, _llp, _dp, ctypes.c_int], ctypes.c_int),
    "gbs_queue_run": ([_vp, _vp], ctypes.c_int),
    "gbs_session_set_graphs": ([_vp, ctypes.c_int], ctypes.c_int),
    "gbs_set_split": ([ctypes.c_int] * 5, ctypes.c_int),
    "gbs_get_split": ([ctypes.c_int, ctypes.c_int, ctypes.c_int, _ip, _ip], ctypes.c_int),
    "gbs_queue_read": ([_vp, _vp, _dp, _dp, _ip], ctypes.c_int),
    "gbs_lhaf_repeated_host": ([_dp, _dp, ctypes.c_int, _ip, ctypes.c_int, _dp], ctypes.c_int),
    "gbs_lhaf_repeated_cert_host": ([_dp, _dp, ctypes.c_int, _ip, ctypes.c_int, _dp, _dp], ctypes.c_int),
    "gbs_sampler_sample": ([_dp, ctypes.c_int, _ip, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, _dp,
                            ctypes.c_ulonglong, _ip], ctypes.c_int),
    "gbs_sampler_conditional_weights": ([_dp, ctypes.c_int, _ip, ctypes.c_int, ctypes.c_int, _ip, ctypes.c_int,
                                         ctypes.c_int, _dp], ctypes.c_int),
    "gbs_sampler_last_error": ([], ctypes.c_char_p),
    "gbs_sampler_set_dedup": ([ctypes.c_int], ctypes.c_int),
    "gbs_lhaf_repeated_last_error": ([], ctypes.c_char_p),
    "gbs_probe_fp64_peak": ([_dp, ctypes.POINTER(ctypes.c_float)], ctypes.c_int),
    "gbs_probe_fp64_mma": ([ctypes.c_int, _dp, ctypes.POINTER(ctypes.c_float)], ctypes.c_int),
    "gbs_probe_fp64_mma_chains": ([ctypes.c_int] * 4 + [_dp, _dp], ctypes.c_int),
    "gbs_haf_noalloc": ([_vp, ctypes.c_int, ctypes.c_int, _vp, _vp], ctypes.c_int),
    "gbs_haf_noalloc_last_error": ([], ctypes.c_char_p),
}

_LIB = None
_LOAD_ERROR: str | None = None


def load():
    """Load libgbs_b200.so (once).  Raises RuntimeError when it is unavailable."""
    global _LIB, _LOAD_ERROR
    if _LIB is not None:
        return _LIB
    if not LIB_PATH.exists():
        _LOAD_ERROR = f"{LIB_PATH} is not built (run `python -m gbskernels_b200.build`)"
        raise RuntimeError(_LOAD_ERROR)
    try:
        lib = ctypes.CDLL(str(LIB_PATH))
    except OSError as e:  # pragma: no cover - depends on the machine
        _LOAD_ERROR = f"cannot load {LIB_PATH}: {e}"
        raise RuntimeError(_LOAD_ERROR) from e
    for name, (argt, rest) in SIGNATURES.items():
        fn = getattr(lib, name, None)
        if fn is None:
            continue
        fn.argtypes = argt
        fn.restype = rest
    _LIB = lib
    return lib


def exported_symbols() -> list[str]:
    lib = load()
    return [n for n in SIGNATURES if hasattr(lib, n)]


def last_error() -> str:
    lib = load()
    msg = lib.gbs_last_error()
    return msg.decode() if msg else ""


def check(rc: int, what: str) -> None:
    if rc != 0:
        raise RuntimeError(f"{what} failed (code {rc}): {last_error()}")


def dptr(a: np.ndarray):
    return a.ctypes.data_as(_dp)


def iptr(a: np.ndarray):
    return a.ctypes.data_as(_ip)


def llptr(a: np.ndarray):
    return a.ctypes.data_as(_llp)


def device_count() -> int:
    """Number of CUDA devices visible through torch (0 without a GPU)."""
    try:
        import torch
        return torch.cuda.device_count() if torch.cuda.is_available() else 0
    except Exception:  # pragma: no cover
        return 0


def env_flag(name: str) -> bool:
    return os.environ.get(name, "").strip() not in ("", "0", "false", "False")
