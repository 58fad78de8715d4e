"""The reference's own Python package over gbskernels_b200/ext/gbskernels_ext.py, on
the CPU.

The reference loads its GPU extension from $GBSKERNELS_EXT_DIR
(gbskernels/__init__.py:109-136).  This test points it at this repository's
extension module and runs the reference's public API (backend="gpu") in every
tier.  Without a GPU the module's ctypes library is swapped for a fake whose
``gbs_*`` functions read the same pointers and sizes and answer with the oracle,
so what is checked here is the boundary itself: names, argument order, the
dimension argument (matrix side vs mode count), return shapes, the resident
session, the certified ladder and the odd loop-hafnian augmentation the reference
performs before calling.  The same module over the real library is covered on
the GPU by tests/test_gpu_ext_stub.py.

Needs a checkout of the reference (GBS_REFERENCE_DIR, or the build container's
mount); skipped where none exists.
"""

from __future__ import annotations

import os
import subprocess
import sys
import textwrap
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
EXT_DIR = ROOT / "gbskernels_b200" / "ext"
REF = Path(os.environ.get("GBS_REFERENCE_DIR", "/root/reference"))

pytestmark = pytest.mark.skipif(not (REF / "gbskernels" / "__init__.py").exists(),
                                reason="no reference checkout")

_HEAD = "import os, sys\nROOT, REF = sys.argv[1], sys.argv[2]\n"

_FAKE = textwrap.dedent(r'''
    import ctypes
    import numpy as np
    sys.path.insert(0, ROOT)
    import oracle

    def arr(p, n):
        return np.ctypeslib.as_array(p, shape=(n,))

    def cstack(p, d, B):
        return arr(p, 2 * B * d * d).view(np.complex128).reshape(B, d, d)

    def put(p, vals):
        v = np.asarray(vals, np.complex128)
        arr(p, 2 * len(v))[:] = v.view(np.float64)

    class Fake:
        calls = []
        def __getattr__(self, name):
            fn = getattr(self, "_" + name, None)
            if fn is None:
                raise AttributeError(name)
            def wrapped(*a):
                Fake.calls.append(name)
                return fn(*[x.value if isinstance(x, ctypes.c_int) else x for x in a])
            return wrapped

        # one-shot batches: (mats, dim_or_modes, batch, out[, aux])
        def _batch(self, func, tier, p, k, B, out, aux=None):
            d = 2 * k if func == "tor" else k
            S = cstack(p, d, B)
            ev = getattr(oracle, func)
            vals, auxv = [], []
            for m in S:
                m = np.real(m) if func == "tor" and not np.any(np.imag(m)) else m
                q = complex(ev(m, "quad"))
                f, absn = ev(m, "fp64", with_absnorm=True)
                if tier == "fp64": vals.append(f)
                elif tier == "dd": vals.append(q)
                elif tier == "kappa": vals.append(f); auxv.append(absn)
                elif tier == "cert":   # a loose but valid enclosure: forces the ladder
                    vals.append(f); auxv.append(abs(f - q) + 1e-3 * abs(q))
                elif tier == "certdd":
                    vals.append(q); auxv.append(1e-15 * abs(q) + 1e-300)
            put(out, vals)
            if aux is not None:
                arr(aux, B)[:] = auxv
            return 0

    for func in ("perm", "haf", "lhaf", "tor"):
        for suffix, tier in (("_host", "fp64"), ("_dd_host", "dd"), ("_kappa_host", "kappa"),
                             ("_certified_host", "cert"), ("_dd_certified_host", "certdd")):
            setattr(Fake, f"_gbs_{func}{suffix}",
                    (lambda f, t: lambda self, *a: self._batch(f, t, *a))(func, tier))

    def _single(self, tier, p, n, g, v, e=None):
        O = arr(p, 4 * n * n).reshape(2 * n, 2 * n).copy()
        q = complex(oracle.tor(O, "quad")).real
        v._obj.value = q
        if e is not None:
            e._obj.value = 1e-14 * abs(q) if tier == "cert" else 1e-20 * abs(q)
        return 0
    Fake._gbs_tor_recursive_single_host = lambda self, *a: _single(self, "fp64", *a)
    Fake._gbs_tor_single_certified_host = lambda self, *a: _single(self, "cert", *a)
    Fake._gbs_tor_single_ddcertified_host = lambda self, *a: _single(self, "dd", *a)

    def _rep(self, pA, pg, M, pr, B, out, bnd=None):
        A = arr(pA, 2 * M * M).view(np.complex128).reshape(M, M).copy()
        g = arr(pg, 2 * M).view(np.complex128).copy()
        r = np.ctypeslib.as_array(pr, shape=(B * M,)).reshape(B, M)
        vals = [oracle.lhaf_repeated(A, g, row, "quad") for row in r]
        put(out, vals)
        if bnd is not None:
            arr(bnd, B)[:] = [1e-14 * abs(x) for x in vals]
        return 0
    Fake._gbs_lhaf_repeated_host = _rep
    Fake._gbs_lhaf_repeated_cert_host = _rep

    # sessions: func 0 perm, 1 haf, 2 lhaf, 3 tor; prec 0 fp64, 1 dd; dim = side
    def _open(self, ref):
        ref._obj.value = 1234
        return 0
    def _evaluate(self, s, func, prec, p, d, B, out):
        f = ("perm", "haf", "lhaf", "tor")[func]
        return self._batch(f, "fp64" if prec == 0 else "dd", p, d // 2 if f == "tor" else d, B, out)
    Fake._gbs_session_open = _open
    Fake._gbs_session_evaluate = _evaluate
    Fake._gbs_session_close = lambda self, s: 0
    Fake._gbs_session_reallocs = lambda self, s: 0
    Fake._gbs_last_error = lambda self: b"fake"
''')

_BODY = textwrap.dedent(r'''
    sys.path.insert(0, REF)
    import gbskernels                       # the reference's own package
    ext = gbskernels._load_gpu_ext()
    assert ext is not None and ext.__file__.startswith(os.environ["GBSKERNELS_EXT_DIR"]), ext
    ext._lib = Fake()
    assert gbskernels.gpu_available() and gbskernels.gpu_backend_kind() == "gpu"
    rng = np.random.default_rng(5)

    def sym(B, N):
        X = rng.standard_normal((B, N, N)) + 1j * rng.standard_normal((B, N, N))
        return 0.25 * (X + np.transpose(X, (0, 2, 1)))

    def close(a, b, tol=1e-10):
        a, b = np.asarray(a), np.asarray(b)
        assert np.all(np.abs(a - b) <= tol * np.abs(b)), (a, b)

    H = sym(3, 8)
    close(gbskernels.haf_batched(H, backend="gpu"), [oracle.haf(m, "quad") for m in H])
    close(gbskernels.haf_batched(H, precision="dd", backend="gpu"), [oracle.haf(m, "quad") for m in H], 1e-15)
    L = sym(2, 7)                           # odd N: the reference augments to 8 before calling
    close(gbskernels.lhaf_batched(L, backend="gpu"), [oracle.lhaf(m, "quad") for m in L])
    assert Fake.calls[-1] == "gbs_lhaf_host"
    P = rng.standard_normal((2, 6, 6)) + 1j * rng.standard_normal((2, 6, 6))
    close(gbskernels.perm_batched(P, backend="gpu"), [oracle.perm(m, "quad") for m in P])
    X = rng.standard_normal((6, 6)); S = X @ X.T / 6 + np.eye(6); O = np.eye(6) - np.linalg.inv(S); O = (O + O.T) / 2
    close(gbskernels.tor_batched(O[None], backend="gpu"), [oracle.tor(O, "quad")])
    v, d = gbskernels.haf_batched(H, precision="auto", backend="gpu", return_diagnostics=True)
    assert Fake.calls.count("gbs_haf_kappa_host") == 1 and all("cancellation" in x for x in d)
    # certified: the loose binary64 certificate escalates to the double-double rung
    v, d = gbskernels.haf_batched(H, precision="certified", backend="gpu", return_diagnostics=True, rtol=1e-12)
    assert [x["tier"] for x in d] == ["certified-dd"] * 3, d
    close(v, [oracle.haf(m, "quad") for m in H], 1e-14)
    v, d = gbskernels.tor(O, precision="certified", backend="gpu", return_diagnostics=True)
    assert d["tier"] == "certified-fp64"
    # resident session through the reference's Workspace (ragged: one call per size)
    with gbskernels.Workspace(backend="gpu") as ws:
        rag = [sym(1, 6)[0], sym(1, 8)[0], sym(1, 6)[0]]
        close(ws.haf_batched(rag), [oracle.haf(m, "quad") for m in rag])
    assert Fake.calls.count("gbs_session_evaluate") == 2 and "gbs_session_open" in Fake.calls
    # single-large torontonian, every tier
    close([gbskernels.tor_single(O)], [oracle.tor(O, "quad")])
    v, d = gbskernels.tor_single(O, certified=True)
    assert d["tier"] == "certified-fp64"
    v, d = gbskernels.tor_single(O, dd=True)
    assert d["tier"] == "certified-dd"
    # the repeated-row sieve
    A = sym(1, 4)[0]; g = 0.1 * np.ones(4, np.complex128); reps = np.array([1, 0, 2, 1])
    close([gbskernels.lhaf_repeated(A, g, reps, backend="gpu")], [oracle.lhaf_repeated(A, g, reps, "quad")])
    v, d = gbskernels.lhaf_repeated(A, g, reps, backend="gpu", certified=True)
    assert d["tier"] == "certified-fp64"
    print("ok")
''')


def test_reference_package_runs_on_this_extension(lib):
    script = _HEAD + _FAKE + _BODY
    env = dict(os.environ, GBSKERNELS_EXT_DIR=str(EXT_DIR))
    r = subprocess.run([sys.executable, "-c", script, str(ROOT), str(REF)], cwd=str(ROOT), env=env,
                       capture_output=True, text=True, timeout=600)
    assert r.returncode == 0 and r.stdout.strip().endswith("ok"), r.stderr[-4000:] + r.stdout[-2000:]
