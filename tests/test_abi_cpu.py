"""The C-ABI surface and the host-side argument checks (CPU only, no device calls)."""

from __future__ import annotations

import re
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]


def _declared_symbols() -> list[str]:
    names = []
    for h in (ROOT / "include").glob("*.h"):
        text = re.sub(r"/\*.*?\*/", "", h.read_text(), flags=re.S)
        names += re.findall(r"\b(gbs_[a-z0-9_]+)\s*\(", text)
    return sorted(set(names))


def test_header_declares_the_reference_host_api():
    names = set(_declared_symbols())
    # the reference's core/host_api.cu entry points for this path
    for f in ("perm", "perm_dd", "haf", "haf_dd", "lhaf", "lhaf_dd", "tor", "tor_dd"):
        assert f"gbs_{f}_host" in names
    for f in ("perm", "haf", "lhaf", "tor"):
        assert f"gbs_{f}_kappa_host" in names
    for f in ("open", "evaluate", "evaluate_resident", "close", "reallocs"):
        assert f"gbs_session_{f}" in names
    assert {"gbs_dev_to_host", "gbs_dev_free", "gbs_queue_evaluate"} <= names


def test_library_exports_every_declared_symbol(lib):
    missing = [n for n in _declared_symbols() if not hasattr(lib, n)]
    assert not missing, f"libgbs_b200.so lacks {missing}"


def test_binding_covers_every_declared_symbol():
    from gbskernels_b200 import _lib
    missing = [n for n in _declared_symbols() if n not in _lib.SIGNATURES]
    assert not missing


def test_binding_arity_matches_the_header():
    """Every ctypes signature takes as many arguments as its declaration in
    include/gbs_b200.h (a mismatch would pass garbage through the C ABI)."""
    import re
    from gbskernels_b200 import _lib, sampler, serving  # noqa: F401  (both extend SIGNATURES)
    hdr = (ROOT / "include" / "gbs_b200.h").read_text()
    hdr = re.sub(r"//[^\n]*", "", hdr)
    hdr = re.sub(r"/\*.*?\*/", "", hdr, flags=re.S)
    decls = re.findall(r"\b(?:int|const char\s*\*|void|double|long long|size_t)\s+\**\s*(gbs_\w+)\s*\(([^)]*)\)\s*;",
                       hdr)
    assert set(n for n, _ in decls) == set(_declared_symbols())
    bad = []
    for name, params in decls:
        p = params.strip()
        n = 0 if p in ("", "void") else len(p.split(","))
        argtypes = _lib.SIGNATURES[name][0]
        if argtypes is not None and len(argtypes) != n:
            bad.append((name, n, len(argtypes)))
    assert not bad


def test_library_is_sm100a(lib):
    from gbskernels_b200 import build
    assert "arch=compute_100a,code=sm_100a" in " ".join(build.ARCH)
    assert lib.gbs_version() >= 100


# ---- argument checks that fail before any device work (reference semantics) ----
def test_precision_and_backend_errors(G):
    A = np.eye(4)
    with pytest.raises(ValueError, match="unknown backend"):
        G.haf(A, backend="tpu")
    with pytest.raises(NotImplementedError):
        G.haf(A, backend="cpu")
    with pytest.raises(NotImplementedError, match="CPU only"):
        G.haf(A, precision="ref")
    with pytest.raises(ValueError, match="unknown precision"):
        G.haf(A, precision="fp32")
    with pytest.raises(ValueError, match="return_diagnostics"):
        G.haf(A, precision="certified")
    with pytest.raises(ValueError, match="requires precision='auto' or 'certified'"):
        G.haf(A, return_diagnostics=True)
    with pytest.raises(ValueError, match="rtol"):
        G.haf(A, rtol=1e-3)
    with pytest.raises(ValueError, match="rtol must be finite"):
        G.haf(A, precision="certified", return_diagnostics=True, rtol=-1.0)


def test_shape_and_cap_errors(G):
    with pytest.raises(ValueError, match="uniform"):
        G.haf_batched(np.zeros((2, 3, 4)))
    with pytest.raises(ValueError, match="exceeds"):
        G.perm_batched(np.zeros((1, 29, 29)))
    with pytest.raises(ValueError, match="exceeds"):
        G.haf_batched(np.zeros((1, 34, 34)))
    with pytest.raises(ValueError, match="exceeds"):
        G.lhaf_batched(np.zeros((1, 33, 33)))   # odd N augments to 34
    with pytest.raises(ValueError, match="even"):
        G.tor_batched(np.zeros((1, 3, 3)))
    with pytest.raises(ValueError, match="real-domain"):
        G.tor_batched(np.eye(4)[None] * (0.1 + 0.1j), precision="dd")
    with pytest.raises(ValueError, match="finite"):
        G.haf(np.full((2, 2), np.nan), precision="certified", return_diagnostics=True)


def test_tor_single_contract_errors(G):
    with pytest.raises(ValueError, match="even"):
        G.tor_single(np.zeros((3, 3)))
    with pytest.raises(ValueError, match="cap 64"):
        G.tor_single(np.zeros((66, 66)))
    with pytest.raises(ValueError, match="symmetric"):
        O = np.zeros((4, 4)); O[0, 1] = 0.1
        G.tor_single(O)
    with pytest.raises(ValueError, match="real-domain"):
        G.tor_single(np.eye(4) * 1j * 0.1)


def test_workspace_lifecycle_errors(G):
    ws = G.Workspace()
    with pytest.raises(RuntimeError, match="entered"):
        ws.haf_batched([np.eye(2)])
    ws.close()
    ws.close()  # idempotent
    with pytest.raises(RuntimeError, match="closed"):
        ws.haf_batched([np.eye(2)])
    with pytest.raises(ValueError, match="unknown backend"):
        G.Workspace(backend="tpu")


def test_tuned_split_table(lib):
    import numpy as np
    from gbskernels_b200 import _lib
    s = np.zeros(1, np.int32)
    w = np.zeros(1, np.int32)
    assert lib.gbs_get_split(1, 0, 20, _lib.iptr(s), _lib.iptr(w)) == 0 and (s[0], w[0]) == (-1, 0)
    assert lib.gbs_set_split(1, 3, 20, 6, 2) == 0  # certified shares the binary64 entry
    assert lib.gbs_get_split(1, 0, 20, _lib.iptr(s), _lib.iptr(w)) == 0 and (s[0], w[0]) == (6, 2)
    assert lib.gbs_get_split(1, 1, 20, _lib.iptr(s), _lib.iptr(w)) == 0 and s[0] == -1  # dd separate
    assert lib.gbs_set_split(1, 0, 20, -1, 0) == 0
    assert lib.gbs_set_split(9, 0, 20, 6, 0) != 0 and lib.gbs_set_split(1, 0, 99, 6, 0) != 0


def test_sampler_reduced_A_host_construction():
    # A = X (I - Q^-1): zero for the vacuum; for one squeezed mode (xxpp, hbar = 2)
    # the two diagonal blocks are conjugate, of modulus tanh r
    from gbskernels_b200 import sampler
    assert np.allclose(sampler.reduced_A(np.eye(2), 1), 0.0)
    r = 0.7
    cov = np.diag([np.exp(-2 * r), np.exp(2 * r)])
    A = sampler.reduced_A(cov, 1)
    assert np.allclose(A, A.T)
    assert abs(abs(A[0, 0]) - np.tanh(r)) < 1e-12 and abs(A[1, 1] - np.conj(A[0, 0])) < 1e-12
    assert abs(A[0, 1]) < 1e-12
    with pytest.raises(ValueError):
        sampler.sample_resident(np.eye(10), 4, cutoff=4)  # 2 M cutoff = 40 > 32


def test_dlpack_capsule_release_without_consumer():
    # an unconsumed "dltensor" capsule releases its keep-alive itself
    import gc
    from gbskernels_b200 import _dlpack

    class Owner:
        live = 0

        def _export_acquired(self):
            Owner.live += 1

        def _export_released(self):
            Owner.live -= 1

    c = _dlpack.capsule(Owner(), 0x1000, 5, "<c16", 0)
    assert Owner.live == 1 and len(_dlpack._LIVE) == 1
    del c
    gc.collect()
    assert Owner.live == 0 and not _dlpack._LIVE


def test_missing_library_raises_instead_of_falling_back():
    """Without libgbs_b200.so every GPU entry point raises RuntimeError (no CPU
    fallback), checked in a fresh interpreter with the library path redirected."""
    import subprocess
    import sys
    code = (
        "import sys, numpy as np\n"
        "from pathlib import Path\n"
        "from gbskernels_b200 import _lib\n"
        "_lib.LIB_PATH = Path('does-not-exist') / 'libgbs_b200.so'\n"
        "import gbskernels_b200 as G\n"
        "for call in (lambda: G.haf(np.eye(4)), lambda: G.perm_batched(np.eye(3)[None]),\n"
        "             lambda: G.tor(np.zeros((4, 4)))):\n"
        "    try:\n"
        "        call()\n"
        "    except RuntimeError as e:\n"
        "        assert 'not built' in str(e), e\n"
        "    else:\n"
        "        sys.exit('no error')\n"
        "print('ok')\n")
    r = subprocess.run([sys.executable, "-c", code], cwd=ROOT, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0 and r.stdout.strip() == "ok", r.stderr[-2000:]


def _header_arity() -> dict:
    hdr = (ROOT / "include" / "gbs_b200.h").read_text()
    hdr = re.sub(r"//[^\n]*", "", hdr)
    hdr = re.sub(r"/\*.*?\*/", "", hdr, flags=re.S)
    out = {}
    for name, params in re.findall(
            r"\b(?:int|const char\s*\*|void|double|long long|size_t)\s+\**\s*(gbs_\w+)\s*\(([^)]*)\)\s*;", hdr):
        p = params.strip()
        out[name] = 0 if p in ("", "void") else len(p.split(","))
    return out


def test_extension_module_binds_declared_symbols_with_their_arity(lib):
    """gbskernels_b200/ext/gbskernels_ext.py (the module the reference package
    imports as its extension) names only exported symbols and passes each the
    number of arguments its declaration in include/gbs_b200.h takes."""
    import ast
    src = (ROOT / "gbskernels_b200" / "ext" / "gbskernels_ext.py").read_text()
    tree = ast.parse(src)
    arity = _header_arity()
    named = set()
    for node in ast.walk(tree):
        if not isinstance(node, ast.Call):
            continue
        f = node.func
        # direct calls: _lib.gbs_x(...)
        if isinstance(f, ast.Attribute) and isinstance(f.value, ast.Name) and f.value.id == "_lib":
            named.add(f.attr)
            if f.attr.startswith("gbs_") and not f.attr.endswith("last_error"):
                assert len(node.args) == arity[f.attr], (f.attr, len(node.args), arity[f.attr])
        # table calls: _eval("gbs_x", a) -> (in, dim, batch, out); _eval_aux -> + aux;
        # _tor_single_bound("gbs_x", O, g) -> (O, n, g, out, bound)
        if isinstance(f, ast.Name) and f.id in ("_eval", "_eval_aux", "_tor_single_bound") and node.args \
                and isinstance(node.args[0], ast.Constant):
            name = node.args[0].value
            named.add(name)
            want = {"_eval": 4, "_eval_aux": 5, "_tor_single_bound": 5}[f.id]
            assert arity[name] == want, (name, arity[name], want)
    named = {n for n in named if n.startswith("gbs_")}
    assert len(named) >= 30
    assert all(hasattr(lib, n) for n in named), [n for n in named if not hasattr(lib, n)]
    assert all(n in arity for n in named), [n for n in named if n not in arity]
