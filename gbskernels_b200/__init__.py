"""gbskernels_b200 -- B200-native (sm_100a) batched permanents, hafnians, loop
hafnians and torontonians behind the ``gbskernels`` API of chaofanzhougit/GBSKernels.

Drop-in for the reference's ``backend="gpu"`` path (gbskernels/__init__.py:517-908):
the same function names, signatures, precision tiers, return shapes, diagnostics
dictionaries and exception types.  Everything runs in ``libgbs_b200.so`` (C++ host
runtime + hand-written sm_100a kernels) through its C ABI; this module only
marshals numpy arrays.  There is no CPU backend here and no CPU fallback: the
reference's CPU backend (``backend="cpu"``) and its mpmath tier (``"ref"``) stay
in the reference package.

Precision tiers (as in the reference):
  * ``"fp64"``      binary64 throughout (power trace products on FP64 tensor cores);
  * ``"dd"``        double-double value path;
  * ``"auto"``      fp64 plus the cancellation indicator kappa = sum|term| / |value|,
                    elements with kappa >= 1e8 rerun in double-double ON THE DEVICE
                    (the reference's CPU mpmath rerun does not exist here);
  * ``"certified"`` value plus a rigorous bound |value - exact| <= abs_error_bound.
"""

from __future__ import annotations

import ctypes
from typing import Any, Iterable

import numpy as np

from . import _lib

__version__ = "0.1.0"
__all__ = [
    "perm", "perm_batched", "haf", "haf_batched", "lhaf", "lhaf_batched",
    "tor", "tor_batched", "tor_single", "lhaf_repeated", "gpu_available", "gpu_backend_kind",
    "Workspace", "PRECISIONS", "queue_evaluate", "Server", "serve_stream",
]

PRECISIONS = ("fp64", "ref", "dd", "auto", "certified")
_FN = {"perm": 0, "haf": 1, "lhaf": 2, "tor": 3}
_TIER = {"fp64": 0, "dd": 1, "kappa": 2, "certified": 3, "certified-dd": 4}
_AUTO_KAPPA_MAX = 1e8  # gbskernels/__init__.py:240

# Largest input side each kernel family supports (tor: 2n).
_GPU_MAX_DIM = {
    "perm": 28, "perm_dd": 28,
    "haf": 32, "haf_dd": 32,
    "lhaf": 32, "lhaf_dd": 32,
    "tor": 48, "tor_dd": 48,
}
_TOR_COMPLEX_MAX_DIM = 24  # complex O (subset LU path), the reference's GPU cap


# ------------------------------------------------------------------ helpers
def _check_backend(backend: str) -> None:
    if backend == "gpu":
        return
    if backend == "cpu":
        raise NotImplementedError(
            "gbskernels_b200 implements backend='gpu' only; the CPU backend is the "
            "reference package's cpu_ref")
    raise ValueError(f"unknown backend {backend!r}; expected 'cpu' or 'gpu'")


def _as_stack(matrices: Iterable[Any]) -> np.ndarray:
    stack = np.ascontiguousarray(np.asarray(matrices, dtype=np.complex128))
    if stack.ndim != 3 or stack.shape[1] != stack.shape[2]:
        raise ValueError(
            "GPU backend needs a uniform (B, d, d) stack of square matrices; "
            "ragged batches go through gbskernels_b200.Workspace.")
    return stack


def _prepare(func: str, matrices: Iterable[Any], precision: str) -> np.ndarray:
    """Validate a uniform bucket (gbskernels/__init__.py:158-219 semantics)."""
    if precision not in ("fp64", "dd"):
        if precision == "ref":
            raise NotImplementedError(
                "'ref' is the mpmath ground truth -- CPU only (backend='cpu').")
        raise ValueError(f"unknown precision {precision!r}; expected one of {PRECISIONS}")
    stack = _as_stack(matrices)
    d = int(stack.shape[1])
    name = func if precision == "fp64" else f"{func}_dd"
    deff = d + (d & 1) if func == "lhaf" else d
    if func == "tor" and d % 2:
        raise ValueError("torontonian requires an even dimension 2n")
    if deff > _GPU_MAX_DIM[name]:
        raise ValueError(f"GPU {name}: matrix dimension {d} exceeds the kernel's limit "
                         f"{_GPU_MAX_DIM[name]}")
    if func == "tor" and stack.size and float(np.max(np.abs(stack.imag))) > 0.0:
        if precision == "dd":
            raise ValueError("GPU torontonian (precision='dd') is real-domain only; the input "
                             "has non-zero imaginary parts.")
        if d > _TOR_COMPLEX_MAX_DIM:
            raise ValueError(f"GPU torontonian of a complex O (subset LU): dimension {d} exceeds "
                             f"the limit {_TOR_COMPLEX_MAX_DIM}")
    return stack


def _is_complex_tor(func: str, stack: np.ndarray) -> bool:
    return func == "tor" and stack.size > 0 and float(np.max(np.abs(stack.imag))) > 0.0


def _kernel_dim(func: str, d: int) -> int:
    return d // 2 if func == "tor" else d


def _call_uniform(func: str, stack: np.ndarray, precision: str) -> np.ndarray:
    lib = _lib.load()
    B, d = stack.shape[0], stack.shape[1]
    out = np.empty(B, dtype=np.complex128)
    if B == 0:
        return out
    name = f"gbs_{func}_host" if precision == "fp64" else f"gbs_{func}_dd_host"
    fn = getattr(lib, name)
    rc = fn(_lib.dptr(stack.view(np.float64)), _kernel_dim(func, d), B, _lib.dptr(out.view(np.float64)))
    _lib.check(rc, name)
    return out


# ------------------------------------------------------------------ tiers
_NOT_SUPPORTED = 801  # cudaErrorNotSupported: a (function, tier) the kernels refuse


def _raise_for(rc: int, what: str, invalid=ValueError, unsupported=ValueError) -> None:
    """Map a library return code to the exception the API contract names: bad
    arguments (code 1) and refused combinations (code 801) become `invalid` /
    `unsupported`, anything else (a CUDA failure) RuntimeError."""
    if rc == 0:
        return
    msg = _lib.last_error()
    if rc == 1:
        raise invalid(f"{what}: {msg}")
    if rc == _NOT_SUPPORTED:
        raise unsupported(f"{what}: {msg}")
    raise RuntimeError(f"{what} failed (code {rc}): {msg}")


def _auto_batched(func: str, matrices, return_diagnostics: bool):
    """fp64 + cancellation indicator, double-double rerun of the elements with
    kappa >= 1e8 -- one library call (gbs_auto_host)."""
    stack = _prepare(func, matrices, "fp64")
    B, d = stack.shape[0], stack.shape[1]
    out = np.empty(B, dtype=np.complex128)
    kappa = np.empty(B, dtype=np.float64)
    tier = np.zeros(B, dtype=np.int32)
    if B:
        rc = _lib.load().gbs_auto_host(_FN[func], _lib.dptr(stack.view(np.float64)), d, B, _AUTO_KAPPA_MAX,
                                       _lib.dptr(out.view(np.float64)), _lib.dptr(kappa), _lib.iptr(tier))
        # a complex torontonian whose indicator asks for the (real-domain) dd rerun
        _raise_for(rc, f"precision='auto' {func}")
    if not return_diagnostics:
        return out
    return out, [{"tier": ("fp64", "dd")[t], "cancellation": float(k)} for t, k in zip(tier, kappa)]


def _certified_batched(func: str, matrices, rtol: float | None):
    """Certified values and bounds; with `rtol`, the proven ladder certified-fp64 ->
    certified-dd runs inside the library (gbs_certified_ladder_host).  An element no
    rung certifies raises FloatingPointError (the reference's mpmath rung is
    CPU-only)."""
    stack = _prepare(func, matrices, "fp64")
    B, d = stack.shape[0], stack.shape[1]
    out = np.empty(B, dtype=np.complex128)
    bound = np.empty(B, dtype=np.float64)
    tier = np.zeros(B, dtype=np.int32)
    if B:
        rc = _lib.load().gbs_certified_ladder_host(_FN[func], _lib.dptr(stack.view(np.float64)), d, B,
                                                   -1.0 if rtol is None else float(rtol),
                                                   _lib.dptr(out.view(np.float64)), _lib.dptr(bound),
                                                   _lib.iptr(tier))
        _raise_for(rc, f"certified {func}", unsupported=NotImplementedError)
    bad = np.flatnonzero(tier < 0)
    if bad.size:
        i = int(bad[0])
        if rtol is None:
            raise FloatingPointError(f"certified {func} batch element {i} refused with a non-finite value or bound")
        raise FloatingPointError(f"certified {func} element {i}: neither the fp64 nor the double-double "
                                 f"certificate reaches rtol={rtol} (the mpmath rung is CPU-only)")
    mag = np.abs(out)
    with np.errstate(divide="ignore", invalid="ignore"):
        rel = np.where(mag > 0, bound / np.where(mag > 0, mag, 1.0), np.where(bound == 0, 0.0, np.inf))
    diags = []
    for t, e, r in zip(tier, bound, rel):
        dg = {"tier": "certified-dd" if t == _TIER["certified-dd"] else "certified-fp64",
              "abs_error_bound": float(e), "rel_error_bound": float(r)}
        if rtol is not None:
            dg["escalated"] = bool(t == _TIER["certified-dd"])
        diags.append(dg)
    return out, diags


def _validate_options(precision, return_diagnostics, rtol) -> None:
    """The API's option contract: diagnostics exist for the auto and certified tiers
    only and the certified tier must return them (its bound is the point of it);
    rtol belongs to the certified tier and is a finite non-negative number."""
    if return_diagnostics and precision not in ("auto", "certified"):
        raise ValueError("return_diagnostics=True requires precision='auto' or 'certified'")
    if precision == "certified" and not return_diagnostics:
        raise ValueError("precision='certified' reports the bound of its certificate in the diagnostics: "
                         "pass return_diagnostics=True")
    if rtol is None:
        return
    if precision != "certified":
        raise ValueError("rtol is a parameter of precision='certified'")
    if not np.isfinite(rtol) or rtol < 0.0:
        raise ValueError("rtol must be finite and non-negative")


def _dispatch_batched(func, matrices, precision, backend, return_diagnostics=False, rtol=None):
    _validate_options(precision, return_diagnostics, rtol)
    _check_backend(backend)
    if precision == "auto":
        return _auto_batched(func, matrices, return_diagnostics)
    if precision == "certified":
        return _certified_batched(func, matrices, rtol)
    stack = _prepare(func, matrices, precision)
    return _call_uniform(func, stack, precision)


def _dispatch_single(func, A, precision, backend, return_diagnostics=False, rtol=None):
    res = _dispatch_batched(func, np.asarray(A)[None, ...], precision, backend, return_diagnostics, rtol)
    if isinstance(res, tuple):
        vals, diags = res
        return complex(vals[0]), diags[0]
    return complex(res[0])


# ------------------------------------------------------------------ public API
def perm(A: Any, precision: str = "fp64", backend: str = "gpu", return_diagnostics: bool = False,
         rtol: float | None = None):
    """Permanent of a single square matrix ``A``."""
    return _dispatch_single("perm", A, precision, backend, return_diagnostics, rtol)


def perm_batched(matrices: Iterable[Any], precision: str = "fp64", backend: str = "gpu",
                 return_diagnostics: bool = False, rtol: float | None = None):
    """Permanents of a (B, n, n) batch -> complex128 vector."""
    return _dispatch_batched("perm", matrices, precision, backend, return_diagnostics, rtol)


def haf(A: Any, precision: str = "fp64", backend: str = "gpu", return_diagnostics: bool = False,
        rtol: float | None = None):
    """Hafnian of a single symmetric matrix (diagonal ignored)."""
    return _dispatch_single("haf", A, precision, backend, return_diagnostics, rtol)


def haf_batched(matrices: Iterable[Any], precision: str = "fp64", backend: str = "gpu",
                return_diagnostics: bool = False, rtol: float | None = None):
    """Hafnians of a (B, N, N) batch of symmetric matrices -> complex128 vector."""
    return _dispatch_batched("haf", matrices, precision, backend, return_diagnostics, rtol)


def lhaf(A: Any, precision: str = "fp64", backend: str = "gpu", return_diagnostics: bool = False,
         rtol: float | None = None):
    """Loop hafnian of a single symmetric matrix (odd N via A (+) [1])."""
    return _dispatch_single("lhaf", A, precision, backend, return_diagnostics, rtol)


def lhaf_batched(matrices: Iterable[Any], precision: str = "fp64", backend: str = "gpu",
                 return_diagnostics: bool = False, rtol: float | None = None):
    """Loop hafnians of a (B, N, N) batch -> complex128 vector."""
    return _dispatch_batched("lhaf", matrices, precision, backend, return_diagnostics, rtol)


def tor(O: Any, precision: str = "fp64", backend: str = "gpu", return_diagnostics: bool = False,
        rtol: float | None = None):
    """Torontonian of a single 2n x 2n matrix O (xxpp ordering)."""
    return _dispatch_single("tor", O, precision, backend, return_diagnostics, rtol)


def tor_batched(matrices: Iterable[Any], precision: str = "fp64", backend: str = "gpu",
                return_diagnostics: bool = False, rtol: float | None = None):
    """Torontonians of a (B, 2n, 2n) batch -> complex128 vector."""
    return _dispatch_batched("tor", matrices, precision, backend, return_diagnostics, rtol)


def lhaf_repeated(A: Any, gamma: Any, reps: Any, backend: str = "gpu", certified: bool = False):
    """Loop hafnians of ``A`` expanded by repetition patterns
    (gbskernels/__init__.py:561-632 contract).

    ``A`` is the (M, M) base matrix, ``gamma`` the length-M loop weights (``None`` ->
    zeros: the ordinary hafnian of the expansion), ``reps`` a (B, M) table of
    non-negative counts (or one length-M pattern).  Returns the (B,) values (a scalar
    for one pattern) of the finite-difference sieve, ``prod(n_i + 1)`` terms per
    pattern, evaluated on the GPU (``libgbs_b200`` sieve kernel).  Caps: M <= 32,
    sum(reps) <= 64, prod(n_i + 1) <= 2^40.  ``certified=True``: values bit-identical
    to the plain sieve plus a rigorous per-pattern bound; returns ``(values,
    {"tier": "certified-fp64", "abs_error_bound": bounds})`` and raises
    FloatingPointError when a pattern cannot be certified."""
    _check_backend(backend)
    A = np.ascontiguousarray(A, dtype=np.complex128)
    if A.ndim != 2 or A.shape[0] != A.shape[1]:
        raise ValueError(f"lhaf_repeated: A must be square (M, M), got {A.shape}")
    M = A.shape[0]
    g = (np.zeros(M, dtype=np.complex128) if gamma is None
         else np.ascontiguousarray(gamma, dtype=np.complex128))
    if g.shape != (M,):
        raise ValueError(f"lhaf_repeated: gamma must be a length-{M} vector, got {g.shape}")
    r = np.ascontiguousarray(reps, dtype=np.int32)
    single = r.ndim == 1
    if single:
        r = r[None, :]
    if r.ndim != 2 or r.shape[1] != M:
        raise ValueError(f"lhaf_repeated: reps must be (B, {M}) or ({M},), got {np.asarray(reps).shape}")
    if (r < 0).any():
        raise ValueError("lhaf_repeated: reps must be non-negative")
    if M > 32:
        raise ValueError(f"lhaf_repeated: M = {M} exceeds the cap 32")
    if r.size and int(r.sum(axis=1).max()) > 64:
        raise ValueError("lhaf_repeated: sum(reps) exceeds the cap 64")
    B = r.shape[0]
    out = np.empty(B, dtype=np.complex128)
    bounds = np.zeros(B, dtype=np.float64)
    if B:
        lib = _lib.load()
        if certified:
            rc = lib.gbs_lhaf_repeated_cert_host(_lib.dptr(A.view(np.float64)), _lib.dptr(g.view(np.float64)), M,
                                                 _lib.iptr(r), B, _lib.dptr(out.view(np.float64)),
                                                 _lib.dptr(bounds))
        else:
            rc = lib.gbs_lhaf_repeated_host(_lib.dptr(A.view(np.float64)), _lib.dptr(g.view(np.float64)), M,
                                            _lib.iptr(r), B, _lib.dptr(out.view(np.float64)))
        if rc != 0:
            msg = lib.gbs_lhaf_repeated_last_error()
            raise (ValueError if rc == 1 else RuntimeError)(
                f"lhaf_repeated failed (code {rc}): {msg.decode() if msg else ''}")
    if certified:
        valid = (np.all(np.isfinite(out.real)) and np.all(np.isfinite(out.imag))
                 and np.all(np.isfinite(bounds)) and np.all(bounds >= 0.0))
        if not valid:
            raise FloatingPointError("certified lhaf_repeated refused with a non-finite value or bound")
        diag = {"tier": "certified-fp64", "abs_error_bound": float(bounds[0]) if single else bounds}
        return (complex(out[0]) if single else out), diag
    return complex(out[0]) if single else out


def tor_single(O: Any, groups: int | None = None, certified: bool = False, dd: bool = False):
    """Single large torontonian of a real (2n, 2n) matrix, 2n <= 64
    (gbskernels/__init__.py:635-691 contract).

    One instance split into at least ``2**groups`` prefix work items over the
    whole GPU (the warp-cooperative walk of the batched kernel, lifted to 32
    modes).  ``certified=True`` returns ``(value, diagnostics)`` with a rigorous
    a-posteriori bound; ``dd=True`` (implies certified) computes the value in
    double-word arithmetic with the same kind of bound (tier ``"certified-dd"``)."""
    A = np.asarray(O)
    if np.iscomplexobj(A):
        if np.any(np.imag(A) != 0):
            raise ValueError("tor_single is real-domain only; use tor() for complex O (dim <= 24)")
        A = np.real(A)
    M = np.ascontiguousarray(A, dtype=np.float64)
    if M.ndim != 2 or M.shape[0] != M.shape[1] or M.shape[0] % 2 != 0:
        raise ValueError(f"tor_single: O must be square with even dimension, got {M.shape}")
    if M.shape[0] > 64:
        raise ValueError(f"tor_single: dimension {M.shape[0]} exceeds the cap 64 (n <= 32 modes)")
    if not np.all(np.isfinite(M)):
        raise ValueError("tor_single: O must contain only finite binary64 values")
    if not np.array_equal(M, M.T):
        raise ValueError("tor_single: O must be exactly symmetric after conversion to binary64")
    n = M.shape[0] // 2
    g = min(n, 14) if groups is None else int(groups)
    if not 0 <= g <= n:
        raise ValueError(f"groups must be in [0, {n}]")
    lib = _lib.load()
    v = np.zeros(1)
    e = np.zeros(1)
    if certified or dd:
        tier = "certified-dd" if dd else "certified-fp64"
        name = "gbs_tor_single_ddcertified_host" if dd else "gbs_tor_single_certified_host"
        fn = getattr(lib, name, None)
        if fn is None:
            raise RuntimeError(f"tor_single({tier}): the loaded libgbs_b200.so lacks {name}")
        _lib.check(fn(_lib.dptr(M), n, g, _lib.dptr(v), _lib.dptr(e)), name)
        vv, ee = float(v[0]), float(e[0])
        if not (np.isfinite(vv) and np.isfinite(ee) and ee >= 0.0):
            raise ValueError("tor_single: off the physical domain or uncertifiable "
                             "(the bound refuses rather than overclaims)")
        rel = ee / abs(vv) if vv != 0 else float("inf")
        return vv, {"tier": tier, "abs_error_bound": ee, "rel_error_bound": rel}
    fn = getattr(lib, "gbs_tor_recursive_single_host", None)
    if fn is None:
        raise RuntimeError("tor_single: the loaded libgbs_b200.so lacks gbs_tor_recursive_single_host")
    _lib.check(fn(_lib.dptr(M), n, g, _lib.dptr(v)), "gbs_tor_recursive_single_host")
    vv = float(v[0])
    if not np.isfinite(vv):
        raise ValueError("tor_single: input is off the physical domain (I - O_S not SPD)")
    return vv


def gpu_available() -> bool:
    """True if libgbs_b200.so loads and a CUDA device is visible."""
    try:
        _lib.load()
    except RuntimeError:
        return False
    return _lib.device_count() > 0


def gpu_backend_kind() -> str:
    """'gpu' when the sm_100a library loads and a device is present, else 'none'."""
    return "gpu" if gpu_available() else "none"


# ------------------------------------------------------------------ sessions / ragged batches
class _ResidentView:
    """A typed part (aux or status) of a resident result block, on the device."""

    def __init__(self, owner: "_ResidentResult", byte_offset: int, n: int, typestr: str, dtype):
        self._owner = owner
        self._off = byte_offset
        self._n = n
        self._typestr = typestr
        self._dtype = dtype

    @property
    def __cuda_array_interface__(self):
        base = ctypes.cast(self._owner._ptr, ctypes.c_void_p).value or 0
        return {"shape": (self._n,), "typestr": self._typestr, "data": (base + self._off if base else 0, False),
                "version": 3}

    def __dlpack__(self, stream=None):
        from . import _dlpack
        return _dlpack.capsule(self._owner, self._owner._addr() + self._off, self._n, self._typestr,
                               self._owner._device())

    def __dlpack_device__(self):
        return (2, self._owner._device())

    def numpy(self) -> np.ndarray:
        out = np.empty(self._n, dtype=self._dtype)
        if self._n:
            if not self._owner._ptr:
                raise RuntimeError("resident result is closed")
            base = ctypes.cast(self._owner._ptr, ctypes.c_void_p).value
            _lib.check(_lib.load().gbs_dev_copy_to_host(ctypes.c_void_p(base + self._off),
                                                        out.ctypes.data_as(ctypes.c_void_p), out.nbytes),
                       "gbs_dev_copy_to_host")
        return out

    def __len__(self) -> int:
        return self._n


class _ResidentResult:
    """Device-resident (B,) complex128 result (gbskernels/__init__.py:856-908 contract).
    Exposes ``__cuda_array_interface__`` so ``torch.as_tensor(r, device='cuda')`` or
    CuPy consume it without a copy; ``.numpy()`` copies to the host.  The block also
    holds, on the device, ``.aux`` (float64: the certified bound, the indicator sum
    or kappa, by tier) and ``.status`` (int32, 0 = ok; the value is NaN otherwise)."""

    def __init__(self, ptr: ctypes.POINTER(ctypes.c_double), n: int):
        self._ptr = ptr
        self._n = n
        self._exports = 0            # live DLPack tensors over this block
        self._close_pending = False
        self._dev = None
        self.aux = _ResidentView(self, 16 * n, n, "<f8", np.float64)
        self.status = _ResidentView(self, 24 * n, n, "<i4", np.int32)

    def _addr(self) -> int:
        if not self._ptr:
            raise RuntimeError("resident result is closed")
        return ctypes.cast(self._ptr, ctypes.c_void_p).value

    def _device(self) -> int:
        if self._dev is None:
            d = np.zeros(1, np.int32)
            _lib.check(_lib.load().gbs_dev_device(ctypes.c_void_p(self._addr()), _lib.iptr(d)), "gbs_dev_device")
            self._dev = int(d[0])
        return self._dev

    def _export_acquired(self) -> None:
        self._exports += 1

    def _export_released(self) -> None:
        self._exports -= 1
        if self._exports == 0 and self._close_pending:
            self._close_pending = False
            self.close()

    @property
    def __cuda_array_interface__(self):
        addr = ctypes.cast(self._ptr, ctypes.c_void_p).value or 0
        return {"shape": (self._n,), "typestr": "<c16", "data": (addr, False), "version": 3}

    def __dlpack__(self, stream=None):
        """DLPack capsule of the (B,) complex128 values on the device (no copy; the
        results are complete when the handle is returned, so any stream may read)."""
        from . import _dlpack
        return _dlpack.capsule(self, self._addr(), self._n, "<c16", self._device())

    def __dlpack_device__(self):
        return (2, self._device())  # kDLCUDA

    def numpy(self) -> np.ndarray:
        out = np.empty(self._n, dtype=np.complex128)
        if self._n:
            if not self._ptr:
                raise RuntimeError("resident result is closed")
            _lib.check(_lib.load().gbs_dev_to_host(self._ptr, _lib.dptr(out.view(np.float64)), self._n),
                       "gbs_dev_to_host")
        return out

    def __len__(self) -> int:
        return self._n

    def close(self) -> None:
        """Release the device block (deferred while DLPack tensors over it are alive)."""
        if self._exports > 0:
            self._close_pending = True
            return
        if self._ptr:
            _lib.load().gbs_dev_free(self._ptr)
            self._ptr = None

    def __del__(self):  # pragma: no cover
        try:
            self.close()
        except Exception:
            pass


def _as_square_list(matrices: Iterable[Any]) -> list[np.ndarray]:
    out = []
    for i, m in enumerate(matrices):
        a = np.ascontiguousarray(np.asarray(m, dtype=np.complex128))
        if a.ndim != 2 or a.shape[0] != a.shape[1]:
            raise ValueError(f"Workspace: matrix #{i} must be square 2-D; got shape {a.shape}")
        out.append(a)
    return out


def _pack(mats: list[np.ndarray]) -> tuple[np.ndarray, np.ndarray, np.ndarray]:
    dims = np.array([m.shape[0] for m in mats], dtype=np.int32)
    sizes = dims.astype(np.int64) ** 2
    offsets = np.zeros(len(mats), dtype=np.int64)
    if len(mats) > 1:
        offsets[1:] = np.cumsum(sizes)[:-1]
    buf = np.empty(int(sizes.sum()) if len(mats) else 1, dtype=np.complex128)
    for m, o, s in zip(mats, offsets, sizes):
        buf[o:o + s] = m.reshape(-1)
    return buf, dims, offsets


_C128 = np.dtype(np.complex128)
try:  # the batch walk in C (built beside the library); the Python loop below otherwise
    from . import _hostptr
except ImportError:
    _hostptr = None


def _pointers(mats) -> tuple[np.ndarray, np.ndarray, list]:
    """Host pointer and side of every matrix, for the pointer entry points: a
    C-contiguous complex128 array is passed as it is, anything else is converted
    first (the converted arrays are returned so they outlive the call).  Raises
    ValueError naming the first matrix that is not square 2-D."""
    B = len(mats)
    ptr = np.empty(B, dtype=np.uint64)
    dims = np.empty(B, dtype=np.int32)
    keep = []
    todo = _hostptr.collect(mats, ptr, dims) if _hostptr is not None else range(B)
    for i in todo:
        m = mats[i]
        if not (type(m) is np.ndarray and m.dtype == _C128 and m.flags.c_contiguous):
            m = np.ascontiguousarray(np.asarray(m, dtype=np.complex128))
            keep.append(m)
        sh = m.shape
        if len(sh) != 2 or sh[0] != sh[1]:
            raise ValueError(f"Workspace: matrix #{i} must be square 2-D; got shape {sh}")
        dims[i] = sh[0]
        ptr[i] = m.ctypes.data
    return ptr, dims, keep


class Workspace:
    """Device-resident, bucketing session for ragged, sampler-shaped workloads
    (gbskernels/__init__.py:734-908).  One C++ session (stream, monotonically grown
    device buffers, pinned staging) serves every call.  A ragged batch runs as ONE
    persistent launch over a device work queue (``persistent=True``, default) or as
    one launch per (function, size) bucket (``persistent=False``, the reference's
    plain per-size path); values are identical either way."""

    def __init__(self, backend: str = "gpu", persistent: bool = True) -> None:
        if backend not in ("cpu", "gpu"):
            raise ValueError(f"unknown backend {backend!r}; expected 'cpu' or 'gpu'")
        self._backend = backend
        self._persistent = persistent
        self._session = None
        self._closed = False

    def __enter__(self) -> "Workspace":
        _check_backend(self._backend)
        lib = _lib.load()
        h = ctypes.c_void_p()
        _lib.check(lib.gbs_session_open(ctypes.byref(h)), "gbs_session_open")
        self._session = h
        return self

    def __exit__(self, *exc: Any) -> bool:
        self.close()
        return False

    def close(self) -> None:
        """Release the device-resident session.  Idempotent."""
        if self._closed:
            return
        if self._session is not None:
            _lib.load().gbs_session_close(self._session)
        self._session = None
        self._closed = True

    @property
    def reallocs(self) -> int:
        if self._session is None:
            return 0
        return int(_lib.load().gbs_session_reallocs(self._session))

    def last_stats(self) -> dict:
        ms = np.zeros(1)
        launches = np.zeros(1, dtype=np.int32)
        items = np.zeros(1, dtype=np.int64)
        _lib.check(_lib.load().gbs_session_last_stats(self._session, _lib.dptr(ms), _lib.iptr(launches),
                                                      _lib.llptr(items)), "gbs_session_last_stats")
        return {"kernel_ms": float(ms[0]), "launches": int(launches[0]), "items": int(items[0])}

    def _require(self):
        if self._closed:
            raise RuntimeError("Workspace is closed")
        if self._session is None:
            raise RuntimeError("Workspace must be entered (use `with Workspace() as ws:`)")

    def perm_batched(self, matrices, precision: str = "fp64") -> np.ndarray:
        return self._ragged("perm", matrices, precision)

    def haf_batched(self, matrices, precision: str = "fp64") -> np.ndarray:
        return self._ragged("haf", matrices, precision)

    def lhaf_batched(self, matrices, precision: str = "fp64") -> np.ndarray:
        return self._ragged("lhaf", matrices, precision)

    def tor_batched(self, matrices, precision: str = "fp64") -> np.ndarray:
        return self._ragged("tor", matrices, precision)

    def _ragged(self, func: str, matrices, precision: str) -> np.ndarray:
        """One function over a ragged batch: every size in one persistent launch (the
        auto tier in two: fp64 + indicator, then the double-double reruns).  A
        rejected matrix raises ValueError naming its position."""
        self._require()
        if precision == "ref":
            raise NotImplementedError("'ref' is the mpmath ground truth -- CPU only (backend='cpu').")
        if precision not in ("fp64", "dd", "auto"):
            raise ValueError(f"unknown precision {precision!r} for a ragged batch; expected fp64, dd or auto")
        mats = matrices if isinstance(matrices, list) else list(matrices)
        B = len(mats)
        out = np.empty(B, dtype=np.complex128)
        if B == 0:
            return out
        fns = np.full(B, _FN[func], dtype=np.int32)
        lib = _lib.load()
        if precision != "auto":
            ptr, dims, keep = _pointers(mats)
            tiers = np.full(B, _TIER[precision], dtype=np.int32)
            rc = lib.gbs_queue_evaluate_ptrs(self._session, B, _lib.iptr(fns), _lib.iptr(tiers), _lib.iptr(dims),
                                             ctypes.c_void_p(ptr.ctypes.data), 0 if self._persistent else 1,
                                             _lib.dptr(out.view(np.float64)), None, None)
            del keep
            _raise_for(rc, f"Workspace.{func}_batched")
            return out
        mats = _as_square_list(mats)
        buf, dims, offs = _pack(mats)
        kappa = np.empty(B)
        tier = np.zeros(B, dtype=np.int32)
        rc = lib.gbs_queue_evaluate_auto(self._session, B, _lib.iptr(fns), _lib.iptr(dims), _lib.llptr(offs),
                                         _lib.dptr(buf.view(np.float64)), _AUTO_KAPPA_MAX,
                                         _lib.dptr(out.view(np.float64)), _lib.dptr(kappa), _lib.iptr(tier), None)
        _raise_for(rc, f"Workspace.{func}_batched")
        return out

    def evaluate_full(self, funcs: list[str], mats: list[np.ndarray], precisions: list[str]):
        """As `evaluate`, returning (values, aux, status): aux is sum|term| for the
        'kappa' tier and the rigorous bound for 'certified' (0 otherwise)."""
        self._require()
        B = len(mats)
        out = np.empty(B, dtype=np.complex128)
        st = np.zeros(B, dtype=np.int32)
        aux = np.zeros(B, dtype=np.float64)
        if B:
            self._call_ptrs(funcs, mats, precisions, out, aux, st)
        return out, aux, st

    def _call_ptrs(self, funcs, mats, precisions, out, aux, st) -> None:
        ptr, dims, keep = _pointers(mats)
        fns = np.array([_FN[f] for f in funcs], dtype=np.int32)
        tiers = np.array([_TIER[p] for p in precisions], dtype=np.int32)
        rc = _lib.load().gbs_queue_evaluate_ptrs(
            self._session, len(mats), _lib.iptr(fns), _lib.iptr(tiers), _lib.iptr(dims),
            ctypes.c_void_p(ptr.ctypes.data), 0 if self._persistent else 1,
            _lib.dptr(out.view(np.float64)), _lib.dptr(aux), _lib.iptr(st))
        del keep
        _lib.check(rc, "gbs_queue_evaluate_ptrs")

    def evaluate(self, funcs: list[str], mats: list[np.ndarray], precisions: list[str],
                 return_status: bool = False):
        """Mixed-function, mixed-tier, ragged batch in one persistent launch (or per-size
        launches when the Workspace was opened with persistent=False)."""
        self._require()
        B = len(mats)
        out = np.empty(B, dtype=np.complex128)
        st = np.zeros(B, dtype=np.int32)
        aux = np.zeros(B, dtype=np.float64)
        if B == 0:
            return (out, st) if return_status else out
        self._call_ptrs(funcs, mats, precisions, out, aux, st)
        return (out, st) if return_status else out

    # device-resident outputs (uniform batches)
    def perm_resident(self, matrices, precision: str = "fp64"):
        return self._resident("perm", matrices, precision)

    def haf_resident(self, matrices, precision: str = "fp64"):
        return self._resident("haf", matrices, precision)

    def lhaf_resident(self, matrices, precision: str = "fp64"):
        return self._resident("lhaf", matrices, precision)

    def tor_resident(self, matrices, precision: str = "fp64"):
        return self._resident("tor", matrices, precision)

    def _resident(self, func: str, matrices, precision: str):
        """Uniform batch, result left on the device in request order (every tier:
        fp64, dd, auto -- aux = kappa --, certified -- aux = the bound)."""
        self._require()
        if precision == "ref":
            raise NotImplementedError("'ref' is the mpmath ground truth -- CPU only (backend='cpu').")
        if precision not in ("fp64", "dd", "auto", "certified"):
            raise ValueError(f"unknown precision {precision!r}; expected one of {PRECISIONS}")
        try:
            stack = np.ascontiguousarray(np.asarray(matrices, dtype=np.complex128))
            uniform = stack.ndim == 3
        except (ValueError, TypeError):
            uniform = False
        if not uniform:
            raise ValueError("device-resident output of a ragged batch: use Workspace.evaluate_resident")
        stack = _prepare(func, stack, "dd" if precision == "dd" else "fp64")
        if precision == "auto" and _is_complex_tor(func, stack):
            raise NotImplementedError("auto torontonian of a complex O: the double-double rerun is "
                                      "real-domain only; use precision='fp64'")
        B, d = stack.shape[0], stack.shape[1]
        tier = {"fp64": 0, "dd": 1, "certified": 3, "auto": -1}[precision]
        ptr = ctypes.POINTER(ctypes.c_double)()
        rc = _lib.load().gbs_session_evaluate_resident_tier(self._session, _FN[func], tier,
                                                            _lib.dptr(stack.view(np.float64)), d, B,
                                                            ctypes.byref(ptr))
        _raise_for(rc, f"Workspace.{func}_resident", unsupported=NotImplementedError)
        return _ResidentResult(ptr, B)

    def evaluate_resident(self, funcs: list[str], mats: list[np.ndarray], precisions: list[str] | None = None):
        """Ragged, mixed-function, mixed-tier batch with the results left on the device
        in request order (scattered there; aux and status alongside)."""
        self._require()
        B = len(mats)
        precisions = precisions or ["fp64"] * B
        if not (len(funcs) == B == len(precisions)):
            raise ValueError("funcs, mats and precisions must have the same length")
        if B == 0:
            return _ResidentResult(ctypes.POINTER(ctypes.c_double)(), 0)
        mats = _as_square_list(mats)
        buf, dims, offs = _pack(mats)
        fns = np.array([_FN[f] for f in funcs], dtype=np.int32)
        tiers = np.array([_TIER[p] for p in precisions], dtype=np.int32)
        ptr = ctypes.POINTER(ctypes.c_double)()
        rc = _lib.load().gbs_queue_evaluate_resident(
            self._session, B, _lib.iptr(fns), _lib.iptr(tiers), _lib.iptr(dims), _lib.llptr(offs),
            _lib.dptr(buf.view(np.float64)), 0 if self._persistent else 1, ctypes.byref(ptr))
        _lib.check(rc, "gbs_queue_evaluate_resident")
        return _ResidentResult(ptr, B)


def queue_evaluate(funcs: list[str], mats: list[np.ndarray], precisions: list[str] | None = None,
                   persistent: bool = True) -> np.ndarray:
    """One-shot mixed batch (functions, sizes and fp64/dd tiers mixed) through a
    temporary Workspace."""
    precisions = precisions or ["fp64"] * len(mats)
    with Workspace(persistent=persistent) as ws:
        return ws.evaluate(funcs, [np.asarray(m, dtype=np.complex128) for m in mats], precisions)


from .serving import Server, serve_stream  # noqa: E402
