"""Parity of the sm_100a kernels with the oracle and the reference's golden vectors.

Tolerances: binary64 tiers must be within relative error 1e-10 of the ground truth
(mpmath from the reference, or the binary128 oracle), the double-double tier within
1e-15 (it is collapsed to binary64 at the API), and integer-valued closed forms are
checked to 1e-12.  Reference test models: tests/test_layer1_combinatorial.py,
tests/test_hafnian_layer1.py, tests/test_loop_hafnian.py, tests/test_torontonian.py,
tests/test_layer5_engineering.py, tests/test_precision_auto.py.
"""

from __future__ import annotations

import math

import numpy as np
import pytest

from conftest import golden_cases, rel_err

pytestmark = pytest.mark.gpu

FP64_TOL = 1e-10
DD_TOL = 1e-15
RNG = np.random.default_rng(123)


def sym(N, cplx=True, scale=0.5):
    X = RNG.standard_normal((N, N)) + (1j * RNG.standard_normal((N, N)) if cplx else 0)
    return scale * (X + X.T) / 2


def phys_O(n, scale=1.0):
    X = RNG.standard_normal((2 * n, 2 * n))
    S = scale * X @ X.T / (2 * n) + np.eye(2 * n)
    O = np.eye(2 * n) - np.linalg.inv(S)
    return (O + O.T) / 2


def _batched(G, func):
    return getattr(G, f"{func}_batched")


# ---------------------------------------------------------------- golden vectors
@pytest.mark.parametrize("func", ["perm", "haf", "lhaf", "tor"])
@pytest.mark.parametrize("precision", ["fp64", "dd"])
def test_golden_vectors(gpu, golden, func, precision):
    for m, truth, _, i in golden_cases(golden, func):
        if func == "tor" and np.any(np.imag(m) != 0) and precision == "dd":
            continue  # complex O: the double-double torontonian is real-domain only
        v = _batched(gpu, func)(m[None], precision=precision)[0]
        tol = FP64_TOL if precision == "fp64" else DD_TOL
        if abs(truth) < 1e-6:
            assert abs(v - truth) < 1e-13, (func, i)
        else:
            assert rel_err(v, truth) < tol, (func, precision, i, v, truth)


@pytest.mark.parametrize("func", ["perm", "haf", "lhaf", "tor"])
def test_golden_indicator(gpu, golden, func):
    for m, truth, _, i in golden_cases(golden, func):
        if abs(truth) < 1e-6:
            continue  # kappa is ill-defined at a zero value
        v, diags = _batched(gpu, func)(m[None], precision="auto", return_diagnostics=True)
        absn = golden[f"{func}_absnorm"][i]
        kappa_ref = absn / max(abs(golden[f"{func}_cpu_fp64"][i]), 1e-300)
        assert diags[0]["cancellation"] == pytest.approx(kappa_ref, rel=1e-6), (func, i)
        assert diags[0]["tier"] in ("fp64", "dd")


# ---------------------------------------------------------------- closed forms
@pytest.mark.parametrize("n", [1, 2, 5, 8, 12, 16])
def test_perm_closed_forms(gpu, n):
    assert gpu.perm(np.ones((n, n))) == pytest.approx(math.factorial(n), rel=1e-12)
    assert gpu.perm(np.eye(n)) == pytest.approx(1.0, abs=1e-12)
    A = np.triu(RNG.uniform(-1, 1, (n, n)))
    assert gpu.perm(A) == pytest.approx(np.prod(np.diag(A)), rel=1e-10, abs=1e-14)
    assert gpu.perm(np.ones((n, n)), precision="dd") == pytest.approx(math.factorial(n), rel=1e-15)


@pytest.mark.parametrize("k", [1, 2, 4, 6, 8])
def test_haf_closed_forms(gpu, k):
    N = 2 * k
    dfact = math.prod(range(1, N, 2))
    assert gpu.haf(np.ones((N, N))) == pytest.approx(dfact, rel=1e-12)
    assert gpu.haf(np.ones((N, N)), precision="dd") == pytest.approx(dfact, rel=1e-15)
    blocks = np.zeros((N, N))
    for j in range(k):
        blocks[2 * j, 2 * j + 1] = blocks[2 * j + 1, 2 * j] = j + 1
    assert gpu.haf(blocks) == pytest.approx(math.factorial(k), rel=1e-12)


@pytest.mark.parametrize("N", [1, 2, 3, 6, 9, 12])
def test_lhaf_closed_forms(gpu, N):
    telephone = [1, 1, 2, 4, 10, 26, 76, 232, 764, 2620, 9496, 35696, 140152]
    assert gpu.lhaf(np.ones((N, N))) == pytest.approx(telephone[N], rel=1e-12)
    d = np.linspace(0.5, 1.5, N)
    # the power trace of a diagonal matrix cancels heavily (sum|term| / |value| is
    # 1e5 at N = 12; the reference algorithm in binary64 errs by 6e-12 there)
    v, diag = gpu.lhaf_batched(np.diag(d)[None], precision="auto", return_diagnostics=True)
    kappa = diag[0]["cancellation"]
    assert gpu.lhaf(np.diag(d)) == pytest.approx(np.prod(d), rel=max(1e-13, 1e-15 * kappa))
    a, b, c = 2.0, 3.0, 5.0
    assert gpu.lhaf(np.array([[a, b], [b, c]])) == pytest.approx(b + a * c, rel=1e-14)


@pytest.mark.parametrize("a", [0.05, 0.3, 0.6])
@pytest.mark.parametrize("n", [1, 3, 8])
def test_tor_closed_forms(gpu, a, n):
    assert gpu.tor(a * np.eye(2 * n)) == pytest.approx((a / (1 - a)) ** n, rel=1e-11)
    assert gpu.tor(a * np.eye(2 * n), precision="dd") == pytest.approx((a / (1 - a)) ** n, rel=1e-15)
    assert abs(gpu.tor(np.zeros((2 * n, 2 * n)))) < 1e-12


# ---------------------------------------------------------------- against the oracle at larger sizes
@pytest.mark.parametrize("N", [12, 16, 20])
def test_haf_vs_binary128_oracle(gpu, orc, N):
    mats = np.stack([sym(N), sym(N, cplx=False)])
    for prec, tol in (("fp64", FP64_TOL), ("dd", DD_TOL)):
        got = gpu.haf_batched(mats, precision=prec)
        for i in range(2):
            assert rel_err(got[i], orc.haf(mats[i], "quad")) < tol, (N, prec, i)


@pytest.mark.parametrize("N", [11, 16, 20])
def test_lhaf_vs_binary128_oracle(gpu, orc, N):
    mats = np.stack([sym(N) for _ in range(2)])
    for prec, tol in (("fp64", FP64_TOL), ("dd", DD_TOL)):
        got = gpu.lhaf_batched(mats, precision=prec)
        for i in range(2):
            assert rel_err(got[i], orc.lhaf(mats[i], "quad")) < tol, (N, prec, i)


@pytest.mark.parametrize("N", [2, 4, 5, 6, 8, 9, 10, 12, 14, 16, 18, 20])
def test_real_inputs_vs_binary128_oracle(gpu, orc, N):
    """A real matrix (every imaginary part zero) runs the real power loop (real
    m16n8k8 products, K = s): hafnian (even N) and loop hafnian (odd N augmented)
    against binary128, in fp64 and in the indicator and certified tiers, whose
    values are the fp64 value bit for bit and whose radius encloses the truth."""
    U = 2.0 ** -53
    mats = np.stack([sym(N, cplx=False) for _ in range(3)]).astype(np.complex128)
    funcs = ["lhaf"] if N % 2 else ["haf", "lhaf"]
    for f in funcs:
        fp = _batched(gpu, f)(mats, precision="fp64")
        vk, dk = _batched(gpu, f)(mats, precision="auto", return_diagnostics=True)
        vc, dc = _batched(gpu, f)(mats, precision="certified", return_diagnostics=True)
        for i in range(3):
            t = getattr(orc, f)(mats[i], "quad")
            assert np.imag(fp[i]) == 0.0, (f, N, i)
            assert rel_err(fp[i], t) < FP64_TOL, (f, N, i, fp[i], t)
            if dk[i]["tier"] == "fp64":
                assert vk[i] == fp[i], (f, N, i)
            assert vc[i] == fp[i], (f, N, i)
            assert abs(vc[i] - t) <= dc[i]["abs_error_bound"] * (1 + 1e-12) + U * abs(t), (f, N, i)


@pytest.mark.parametrize("N", [24, 28])
def test_real_inputs_two_strips_vs_oracle_port(gpu, orc, N):
    """Real inputs above 16 (two 16-row strips): against the binary64 oracle port
    of the reference walk, within max(1e-10, 16 N u kappa)."""
    U = 2.0 ** -53
    mats = np.stack([sym(N, cplx=False) for _ in range(2)]).astype(np.complex128)
    for f in ("haf", "lhaf"):
        got = _batched(gpu, f)(mats, precision="fp64")
        for i in range(2):
            v, absn = getattr(orc, f)(mats[i], "fp64", with_absnorm=True)
            tol = max(1e-10, 16 * N * U * absn / abs(v))
            assert rel_err(got[i], v) < tol, (f, N, i, got[i], v, absn / abs(v))


def test_real_and_complex_mixed_equal_alone(gpu):
    """Real and complex instances in one persistent launch: each value bit-identical
    to its evaluation alone (the path is chosen per instance)."""
    mats = [sym(12, cplx=False).astype(complex), sym(12), sym(20, cplx=False).astype(complex), sym(9, cplx=False),
            sym(16), sym(26, cplx=False).astype(complex)]
    funcs = ["haf", "haf", "lhaf", "lhaf", "lhaf", "haf"]
    with gpu.Workspace() as ws:
        together = ws.evaluate(funcs, mats, ["fp64"] * len(mats))
    for i, (f, m) in enumerate(zip(funcs, mats)):
        assert together[i] == _batched(gpu, f)(np.asarray(m, dtype=complex)[None], precision="fp64")[0], i


@pytest.mark.parametrize("n", [13, 16])
def test_perm_vs_binary128_oracle(gpu, orc, n):
    mats = RNG.standard_normal((2, n, n)) + 1j * RNG.standard_normal((2, n, n))
    for prec, tol in (("fp64", FP64_TOL), ("dd", DD_TOL)):
        got = gpu.perm_batched(mats, precision=prec)
        for i in range(2):
            assert rel_err(got[i], orc.perm(mats[i], "quad")) < tol, (n, prec, i)


@pytest.mark.parametrize("n", [6, 11, 14])
def test_tor_vs_binary128_oracle(gpu, orc, n):
    mats = np.stack([phys_O(n) for _ in range(2)])
    for prec, tol in (("fp64", FP64_TOL), ("dd", DD_TOL)):
        got = gpu.tor_batched(mats, precision=prec)
        for i in range(2):
            assert rel_err(got[i], orc.tor(mats[i], "quad")) < tol, (n, prec, i)


# ---------------------------------------------------------------- size-independent properties at full sizes
def test_haf_direct_sum_at_N30(gpu):
    A, B = sym(14), sym(16)
    blk = np.zeros((30, 30), dtype=complex)
    blk[:14, :14], blk[14:, 14:] = A, B
    h = gpu.haf_batched(np.stack([blk]))[0]
    assert rel_err(h, gpu.haf(A) * gpu.haf(B)) < 1e-9


def test_lhaf_direct_sum_at_N28(gpu):
    A, B = sym(12), sym(16)
    blk = np.zeros((28, 28), dtype=complex)
    blk[:12, :12], blk[12:, 12:] = A, B
    assert rel_err(gpu.lhaf(blk), gpu.lhaf(A) * gpu.lhaf(B)) < 1e-9


def test_perm_direct_sum_at_n28(gpu):
    A = RNG.standard_normal((14, 14)) + 1j * RNG.standard_normal((14, 14))
    B = RNG.standard_normal((14, 14)) + 1j * RNG.standard_normal((14, 14))
    blk = np.zeros((28, 28), dtype=complex)
    blk[:14, :14], blk[14:, 14:] = A, B
    assert rel_err(gpu.perm(blk), gpu.perm(A) * gpu.perm(B)) < 1e-9


def test_tor_direct_sum_at_24_modes(gpu):
    O1, O2 = phys_O(12), phys_O(12)
    n1, n2 = 12, 12
    n = n1 + n2
    O = np.zeros((2 * n, 2 * n))
    idx1 = np.r_[0:n1, n:n + n1]
    idx2 = np.r_[n1:n, n + n1:2 * n]
    O[np.ix_(idx1, idx1)] = O1
    O[np.ix_(idx2, idx2)] = O2
    # 2^24 alternating terms cancel (kappa ~ 1e7): the binary64 tier is checked to
    # kappa * 1e-15, the double-double tier to 1e-13
    v, d = gpu.tor(O, precision="auto", return_diagnostics=True)
    prod_dd = gpu.tor(O1, precision="dd") * gpu.tor(O2, precision="dd")
    assert rel_err(gpu.tor(O), prod_dd) < max(1e-10, 1e-15 * d["cancellation"])
    assert rel_err(gpu.tor(O, precision="dd"), prod_dd) < 1e-13


# ---------------------------------------------------------------- edge cases
def test_edge_cases(gpu):
    assert gpu.haf(np.zeros((0, 0))) == 1.0
    assert gpu.haf(np.ones((5, 5))) == 0.0
    assert gpu.perm(np.zeros((0, 0))) == 1.0
    assert gpu.perm(np.array([[3.0 + 1j]])) == 3.0 + 1j
    assert gpu.lhaf(np.array([[7.0]])) == pytest.approx(7.0)
    assert gpu.tor(np.zeros((0, 0))) == 1.0
    for f in ("perm", "haf", "lhaf", "tor"):
        out = _batched(gpu, f)(np.zeros((0, 4, 4)))
        assert out.shape == (0,) and out.dtype == np.complex128


def test_tor_off_domain_gives_nan(gpu):
    O = np.stack([phys_O(3), 1.5 * np.eye(6)])  # second: I - O = -0.5 I not SPD
    v = gpu.tor_batched(O)
    assert np.isfinite(v[0]) and np.isnan(v[1])


# ---------------------------------------------------------------- engineering invariants
@pytest.mark.parametrize("func", ["perm", "haf", "lhaf", "tor"])
def test_batched_equals_looped_bitwise(gpu, func):
    if func == "perm":
        mats = RNG.standard_normal((5, 9, 9)) + 1j * RNG.standard_normal((5, 9, 9))
    elif func == "tor":
        mats = np.stack([phys_O(5) for _ in range(5)])
    else:
        mats = np.stack([sym(10) for _ in range(5)])
    b = _batched(gpu, func)(mats)
    looped = np.array([getattr(gpu, func)(m) for m in mats])
    assert np.array_equal(b, looped)
    assert np.array_equal(b, _batched(gpu, func)(mats))  # deterministic


def test_auto_reruns_cancellation_in_dd(gpu):
    # hafnian family with haf = delta * haf(R): three O(1) matchings cancel to delta
    # (construction of the reference's bench/_inputs.py cancellation_hafnian)
    g = np.random.default_rng(5)
    delta = 1e-9
    Bk = np.array([[0, 1, 1, 1], [1, 0, delta - 2, 1], [1, delta - 2, 0, 1], [1, 1, 1, 0]], dtype=complex)
    G2 = g.standard_normal((4, 4))
    R = G2 + G2.T
    np.fill_diagonal(R, 0)
    A = np.zeros((8, 8), dtype=complex)
    A[:4, :4], A[4:, 4:] = Bk, R
    delta_exact = 2.0 + (delta - 2.0)  # the hafnian of the binary64 block (Sterbenz-exact)
    truth = delta_exact * gpu.haf(R, precision="dd")
    v, d = gpu.haf(A, precision="auto", return_diagnostics=True)
    assert d["tier"] == "dd" and d["cancellation"] >= 1e8
    assert rel_err(v, truth) < 1e-12
    fp = gpu.haf(A)
    assert rel_err(fp, truth) > rel_err(v, truth)


def test_queue_mixed_equals_alone_bitwise(gpu):
    funcs = ["haf", "lhaf", "tor", "haf", "lhaf", "tor", "haf"]
    mats = [sym(8), sym(12), phys_O(5), sym(16), sym(7), phys_O(9), sym(2)]
    precs = ["fp64", "fp64", "fp64", "dd", "kappa", "dd", "fp64"]
    with gpu.Workspace() as ws:
        mixed = ws.evaluate(funcs, mats, precs)
        alone = np.array([ws.evaluate([f], [m], [p])[0] for f, m, p in zip(funcs, mats, precs)])
    with gpu.Workspace(persistent=False) as ws2:
        per_size = ws2.evaluate(funcs, mats, precs)
    assert np.array_equal(mixed, alone)
    assert np.array_equal(mixed, per_size)


def test_wide_launch_equals_narrow_alone_bitwise(gpu):
    # a launch whose largest hafnian has N > 16 runs every subset on the 8-tile code
    # path, one with N <= 16 on the 4-tile path: the values must not depend on it
    rng = np.random.default_rng(2024)  # local: the module stream feeds the other tests

    def lsym(N, scale=0.5):
        X = rng.standard_normal((N, N)) + 1j * rng.standard_normal((N, N))
        return scale * (X + X.T) / 2

    funcs = ["haf", "lhaf", "haf", "lhaf", "haf"]
    mats = [lsym(6), lsym(11), lsym(16), lsym(14), lsym(22)]
    precs = ["fp64", "fp64", "certified", "kappa", "fp64"]
    with gpu.Workspace() as ws:
        mixed = ws.evaluate(funcs, mats, precs)
        alone = np.array([ws.evaluate([f], [m], [p])[0] for f, m, p in zip(funcs, mats, precs)])
    assert np.array_equal(mixed, alone)


def test_workspace_ragged_order_and_reuse(gpu):
    dims = [4, 6, 4, 8, 6, 4, 8]
    mats = [sym(d) for d in dims]
    with gpu.Workspace() as ws:
        got = ws.haf_batched(mats)
        for i, m in enumerate(mats):
            assert got[i] == gpu.haf(m), f"slot {i}"
        r0 = ws.reallocs
        ws.haf_batched(mats[:3])
        assert ws.reallocs == r0  # a smaller batch reuses the resident buffers
        with pytest.raises(ValueError, match="#1"):
            ws.haf_batched([np.eye(4), np.zeros((4, 5))])
        assert ws.haf_batched([]).shape == (0,)


def test_workspace_resident_output(gpu):
    import torch
    mats = np.stack([sym(10) for _ in range(6)])
    with gpu.Workspace() as ws:
        res = ws.haf_resident(mats)
        host = res.numpy()
        t = torch.as_tensor(res, device="cuda")
        assert np.array_equal(host, gpu.haf_batched(mats))
        assert np.array_equal(t.cpu().numpy(), host)
        res.close()


# ---------------------------------------------------------------- complex torontonian (subset LU)
def complex_O(n, scale=0.3):
    X = RNG.standard_normal((2 * n, 2 * n)) + 1j * RNG.standard_normal((2 * n, 2 * n))
    return scale * (X + X.T) / (2 * np.sqrt(2 * n))


@pytest.mark.parametrize("n", [1, 3, 6, 9, 12])
def test_tor_complex_vs_binary128_oracle(gpu, orc, n):
    mats = np.stack([complex_O(n) for _ in range(2)])
    got = gpu.tor_batched(mats)
    for i in range(2):
        truth, absn = orc.tor(mats[i], "quad", with_absnorm=True)
        kappa = absn / abs(truth)  # sum |term| / |tor|
        # each term is a subset LU of a 2m x 2m minor (m <= n): O(n) roundings, so
        # the binary64 sum carries up to ~ n u kappa relative error
        assert rel_err(got[i], truth) < max(FP64_TOL, 4 * n * 2.2e-16 * kappa), (n, i, kappa)
        if kappa < 1e8:  # the auto tier keeps the binary64 value (no double-double rerun)
            v, d = gpu.tor_batched(mats[i:i + 1], precision="auto", return_diagnostics=True)
            assert v[0] == got[i] and d[0]["tier"] == "fp64"
            assert d[0]["cancellation"] == pytest.approx(kappa, rel=1e-6)
        else:
            with pytest.raises(ValueError, match="real-domain"):
                gpu.tor_batched(mats[i:i + 1], precision="auto")


@pytest.mark.parametrize("n", [1, 3, 6, 9])
def test_tor_complex_certified_encloses(gpu, orc, n):
    """Certified tier for a complex O: ball arithmetic through the same subset LU
    (value = the fp64 value bit for bit), the radius enclosing the binary128 LU
    torontonian; there is no double-double rung for a complex O, so an rtol below
    the binary64 certificate is refused."""
    mats = np.stack([complex_O(n) for _ in range(3)])
    fp = gpu.tor_batched(mats)
    v, d = gpu.tor_batched(mats, precision="certified", return_diagnostics=True)
    for i in range(3):
        truth = orc.tor(mats[i], "quad")
        assert v[i] == fp[i]
        assert abs(v[i] - truth) <= d[i]["abs_error_bound"] * (1 + 1e-12), (n, i, d[i])
        assert d[i]["tier"] == "certified-fp64" and np.isfinite(d[i]["abs_error_bound"])
    with pytest.raises(FloatingPointError):
        gpu.tor_batched(mats, precision="certified", return_diagnostics=True, rtol=1e-40)


def test_tor_complex_contract(gpu):
    O = complex_O(4)[None]
    with pytest.raises(ValueError, match="real-domain"):
        gpu.tor_batched(O, precision="dd")
    with pytest.raises(ValueError, match="limit 24"):
        gpu.tor_batched(complex_O(13)[None])
    with gpu.Workspace() as ws:  # ragged mix of real and complex O in one queue
        mats = [complex_O(3), np.real(complex_O(5)), complex_O(2)]
        together = ws.tor_batched(mats)
    alone = np.array([gpu.tor_batched(m[None])[0] for m in mats])
    assert np.array_equal(together, alone)


def test_ragged_auto_equals_each_element_alone(gpu):
    """Workspace auto over a ragged batch (gbs_queue_evaluate_auto: one fp64 +
    indicator launch over every size, one double-double launch of the reruns) gives
    each element the value the uniform auto tier gives it alone."""
    g = np.random.default_rng(9)
    delta = 1e-9
    Bk = np.array([[0, 1, 1, 1], [1, 0, delta - 2, 1], [1, delta - 2, 0, 1], [1, 1, 1, 0]], dtype=complex)
    G2 = g.standard_normal((4, 4))
    R = G2 + G2.T
    np.fill_diagonal(R, 0)
    A = np.zeros((8, 8), dtype=complex)
    A[:4, :4], A[4:, 4:] = Bk, R  # cancels: rerun in double-double
    mats = [sym(6), A, sym(12), sym(6), A.copy(), sym(10)]
    with gpu.Workspace() as ws:
        rag = ws.haf_batched(mats, precision="auto")
    for i, m in enumerate(mats):
        v, d = gpu.haf(m, precision="auto", return_diagnostics=True)
        assert rag[i] == v, i
        assert d["tier"] == ("dd" if m.shape[0] == 8 else "fp64")


def test_pointer_entry_equals_packed_buffer(gpu, lib):
    """gbs_queue_evaluate_ptrs (one host pointer per matrix, the path of
    Workspace.evaluate) gives bit for bit what gbs_queue_evaluate gives from one
    packed buffer: ragged sizes, odd loop hafnians (augmented while packing), a
    permanent and a torontonian, inputs that need converting (a transposed view,
    real float64), every tier; a matrix that is not square is refused by name."""
    import ctypes
    from gbskernels_b200 import _lib
    g = np.random.default_rng(21)
    A16 = sym(16)
    mats = [sym(12), sym(7), A16.T, sym(10).real.copy(), g.standard_normal((9, 9)) + 0j, phys_O(5).astype(complex),
            sym(20), sym(9), sym(14)]
    funcs = ["haf", "lhaf", "haf", "lhaf", "perm", "tor", "lhaf", "lhaf", "haf"]
    for tier_name in ("fp64", "dd", "kappa", "certified"):
        precs = [tier_name] * len(mats)
        with gpu.Workspace() as ws:
            v1, a1, s1 = ws.evaluate_full(funcs, mats, precs)
            conv = [np.ascontiguousarray(np.asarray(m, dtype=np.complex128)) for m in mats]
            buf, dims, offs = gpu._pack(conv)
            B = len(mats)
            v2 = np.empty(B, np.complex128)
            a2 = np.zeros(B)
            s2 = np.zeros(B, np.int32)
            fns = np.array([gpu._FN[f] for f in funcs], np.int32)
            tiers = np.array([gpu._TIER[p] for p in precs], np.int32)
            _lib.check(lib.gbs_queue_evaluate(ws._session, B, _lib.iptr(fns), _lib.iptr(tiers), _lib.iptr(dims),
                                              _lib.llptr(offs), _lib.dptr(buf.view(np.float64)), 0,
                                              _lib.dptr(v2.view(np.float64)), _lib.dptr(a2), _lib.iptr(s2)), "packed")
        assert np.array_equal(v1, v2, equal_nan=True), tier_name
        assert np.array_equal(a1, a2, equal_nan=True), tier_name
        assert np.array_equal(s1, s2), tier_name
    with gpu.Workspace() as ws:
        with pytest.raises(ValueError, match="matrix #1 must be square"):
            ws.evaluate(["haf", "haf"], [sym(6), np.zeros((4, 6), complex)], ["fp64", "fp64"])
        rag_in = [sym(8), sym(12).T, sym(6)]
        ragged = ws.haf_batched(rag_in, precision="dd")
    for i, m in enumerate(rag_in):
        assert ragged[i] == gpu.haf(np.ascontiguousarray(m), precision="dd"), i


def test_certified_ladder_in_library(gpu, lib, orc):
    """gbs_certified_ladder_host: an rtol the binary64 certificate meets keeps it
    (tier 3); a tighter one escalates to the certified double-double rung (tier 4,
    its bound still enclosing the binary128 truth); one that no rung meets is
    refused (tier -1)."""
    import ctypes
    mats = np.stack([sym(12) for _ in range(3)])
    truth = [orc.haf(m, "quad") for m in mats]
    dp = ctypes.POINTER(ctypes.c_double)
    ip = ctypes.POINTER(ctypes.c_int)

    def ladder(rtol):
        out = np.empty(3, np.complex128)
        bnd = np.empty(3)
        tier = np.zeros(3, np.int32)
        rc = lib.gbs_certified_ladder_host(1, mats.ctypes.data_as(dp), 12, 3, rtol, out.ctypes.data_as(dp),
                                           bnd.ctypes.data_as(dp), tier.ctypes.data_as(ip))
        assert rc == 0
        return out, bnd, tier

    for rtol, want in ((1e-3, 3), (1e-14, 4), (1e-30, -1)):
        out, bnd, tier = ladder(rtol)
        assert list(tier) == [want] * 3, (rtol, tier, bnd / np.abs(out))
        if want > 0:
            for i in range(3):
                assert abs(out[i] - truth[i]) <= bnd[i] * (1 + 1e-12) + 1e-300
    v, d = gpu.haf_batched(mats, precision="certified", return_diagnostics=True, rtol=1e-14)
    assert all(x["escalated"] and x["tier"] == "certified-dd" for x in d)
    with pytest.raises(FloatingPointError, match="rtol"):
        gpu.haf_batched(mats, precision="certified", return_diagnostics=True, rtol=1e-30)


@pytest.mark.parametrize("N", [10, 14])
def test_nonsymmetric_input_matches_the_reference_formula(gpu, orc, lib, N):
    """A matrix off symmetry by an antisymmetric E (|E| ~ 1e-9): the reference's
    power trace of the raw entries (n - 1 products; the binary128 oracle) is even in
    E, so it moves by O(|E|^2) only.  The kernels evaluate the symmetric part (the
    half-power identities need B_S symmetric), which must agree with it to the
    tier's accuracy -- a first-order error in E would show at 1e-9 -- and the
    certified double-double radius must enclose it."""
    import ctypes
    g = np.random.default_rng(31)
    A = sym(N)
    X = g.standard_normal((N, N)) + 1j * g.standard_normal((N, N))
    B = A + 1e-9 * (X - X.T)
    np.fill_diagonal(B, 0.3 + 0.1j * np.arange(N) / N)
    for func in ("haf", "lhaf"):
        t = getattr(orc, func)(B, "quad")
        fp = getattr(gpu, f"{func}_batched")(B[None])[0]
        dd = getattr(gpu, f"{func}_batched")(B[None], precision="dd")[0]
        assert rel_err(fp, t) < 1e-12, (func, rel_err(fp, t))
        assert rel_err(dd, t) < 4e-16, (func, rel_err(dd, t))
        out = np.empty(1, np.complex128)
        bnd = np.empty(1)
        dp = ctypes.POINTER(ctypes.c_double)
        Bc = np.ascontiguousarray(B[None])
        assert getattr(lib, f"gbs_{func}_dd_certified_host")(Bc.ctypes.data_as(dp), N, 1, out.ctypes.data_as(dp),
                                                             bnd.ctypes.data_as(dp)) == 0
        # t is the binary128 truth rounded to binary64: its own rounding (<= u|t|) is
        # the slack beside the rigorous radius
        slack = 2.0 ** -53 * abs(t)
        assert abs(out[0] - t) <= bnd[0] * (1 + 1e-12) + slack, (func, abs(out[0] - t), bnd[0])
        v, d = getattr(gpu, f"{func}_batched")(B[None], precision="certified", return_diagnostics=True)
        assert abs(v[0] - t) <= d[0]["abs_error_bound"] + slack, (func, d[0])
