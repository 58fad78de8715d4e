"""Torontonian binary64 tiers (warp-cooperative prefix walk + 32-subset register
tail) at every size class the decomposition distinguishes: k < 5 (tail only), k = 5
(empty prefix), one-item instances, and multi-item instances for both the binary64
decomposition (2^9 leaves per item) and the certified one (2^10), against the
binary128 oracle, the independent double-double kernel (per-lane subtree walk) and
the certified enclosures.  Reference test model: tests/test_torontonian.py and
tests/test_certified.py (tor rows)."""

from __future__ import annotations

import numpy as np
import pytest

from conftest import rel_err

pytestmark = pytest.mark.gpu
RNG = np.random.default_rng(2024)


def phys_O(n, scale=1.0):
    X = RNG.standard_normal((2 * n, 2 * n))
    S = scale * X @ X.T / (2 * n) + np.eye(2 * n)
    O = np.eye(2 * n) - np.linalg.inv(S)
    return (O + O.T) / 2


def _cert(G, mats):
    v, d = G.tor_batched(mats, precision="certified", return_diagnostics=True)
    return v, np.array([x["abs_error_bound"] for x in d])


@pytest.mark.parametrize("n", [1, 2, 4, 5, 6, 7, 9, 10, 12])
def test_tor_sizes_vs_binary128(gpu, orc, n):
    mats = np.stack([phys_O(n), phys_O(n, 3.0)])
    truth = [orc.tor(m, "quad") for m in mats]
    fp = gpu.tor_batched(mats)
    _, diag = gpu.tor_batched(mats, precision="auto", return_diagnostics=True)
    cv, cb = _cert(gpu, mats)
    assert np.array_equal(cv, fp)  # the certified value is the binary64 value
    for i in range(2):
        # sum |term| / |tor| grows like 3^n here: the binary64 error scales with it
        kappa = diag[i]["cancellation"]
        assert rel_err(fp[i], truth[i]) < max(1e-13, 1e-15 * kappa), (n, i, kappa)
        assert abs(cv[i] - truth[i]) <= cb[i], (n, i, abs(cv[i] - truth[i]), cb[i])
        assert cb[i] <= 1e-9 * kappa * abs(truth[i]), (n, i, cb[i] / abs(truth[i]), kappa)


@pytest.mark.parametrize("n", [14, 15, 16, 17])
def test_tor_multi_item_vs_dd_kernel(gpu, n):
    # 14: one work item; 15/16/17: 2/4/8 items (every binary64 tier splits the same
    # way).  The double-double kernel is a separate code path.
    mats = np.stack([phys_O(n) for _ in range(2)])
    _, diag = gpu.tor_batched(mats, precision="auto", return_diagnostics=True)
    dd = gpu.tor_batched(mats, precision="dd")
    f64 = gpu.tor_batched(mats)
    cv, cb = _cert(gpu, mats)
    assert np.array_equal(cv, f64)
    for i in range(2):
        kappa = diag[i]["cancellation"]
        assert rel_err(f64[i], dd[i]) < max(1e-12, 1e-15 * kappa), (n, i, kappa)
        assert abs(cv[i] - dd[i]) <= cb[i], (n, i)
        assert cb[i] <= 1e-9 * kappa * abs(dd[i]), (n, i, cb[i] / abs(dd[i]), kappa)


def test_tor_ragged_batch_equals_alone(gpu):
    sizes = [3, 16, 8, 12, 5, 15, 1]
    mats = [phys_O(n) for n in sizes]
    with gpu.Workspace() as ws:
        together = ws.tor_batched(mats)
    alone = np.array([gpu.tor_batched(m[None])[0] for m in mats])
    assert np.array_equal(together, alone)


def test_tor_certified_non_pd_is_refused(gpu):
    # I - O has a negative eigenvalue: no lower bound on lambda_min can be proved and
    # no subset factorisation may be trusted
    O = phys_O(6)
    w, V = np.linalg.eigh(np.eye(12) - O)
    w[0] = -0.05
    O_bad = np.eye(12) - (V * w) @ V.T
    O_bad = (O_bad + O_bad.T) / 2
    with pytest.raises(FloatingPointError):
        gpu.tor_batched(O_bad[None], precision="certified", return_diagnostics=True)


def test_workload_runner_small_torontonian(gpu):
    from gbskernels_b200 import configs, workloads
    mats = list(workloads.tor_click_batch(16, kmin=10, kmax=14, seed=9))
    res, out, aux, st = configs.run("tor", mats, "certified")
    assert res["status_ok"] == 16 and res["launches"] == 1 and res["kernel_ms"] > 0
    with gpu.Workspace() as ws:
        assert np.array_equal(out, ws.tor_batched(mats))
    assert np.all(aux > 0)


@pytest.mark.parametrize("n", [3, 7, 10, 12])
def test_tor_dd_certified_vs_binary128(gpu, orc, n):
    # the double-double certificate: encloses the binary128 truth and is tight even
    # where the binary64 certificate is loose
    lib = gpu._lib.load()
    mats = np.stack([phys_O(n), phys_O(n, 3.0)])
    cm = np.ascontiguousarray(mats, dtype=np.complex128)
    out = np.empty(2, np.complex128)
    bnd = np.empty(2)
    gpu._lib.check(lib.gbs_tor_dd_certified_host(gpu._lib.dptr(cm.view(np.float64)), n, 2,
                                                 gpu._lib.dptr(out.view(np.float64)), gpu._lib.dptr(bnd)),
                   "gbs_tor_dd_certified_host")
    dd = gpu.tor_batched(mats, precision="dd")
    for i in range(2):
        truth = orc.tor(mats[i], "quad")
        assert abs(out[i] - truth) <= bnd[i], (n, i, abs(out[i] - truth), bnd[i])
        assert bnd[i] <= 1e-14 * abs(truth), (n, i, bnd[i] / abs(truth))
        assert out[i] == dd[i]  # the certified double-double value is the dd value


def test_certified_ladder_escalates_to_dd(gpu):
    from gbskernels_b200 import workloads
    O = np.stack(list(workloads.tor_click_batch(4, kmin=16, kmax=16, seed=8)))
    v, d = gpu.tor_batched(O, precision="certified", return_diagnostics=True, rtol=1e-10)
    dd = gpu.tor_batched(O, precision="dd")
    for i in range(4):
        assert d[i]["rel_error_bound"] <= 1e-10
        if d[i]["tier"] == "certified-dd":
            assert d[i]["escalated"] is True and v[i] == dd[i]
    assert any(x["tier"] == "certified-dd" for x in d)  # click patterns cancel beyond binary64
