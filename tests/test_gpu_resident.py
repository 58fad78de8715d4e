"""Device-resident outputs for every tier and for ragged batches: the results are
scattered to request order on the device; they equal the host-returned values bit
for bit, the aux part carries the tier's extra (bound, indicator sum, kappa) and
torch reads them without a copy (reference contract: gbskernels/__init__.py:856-908,
bindings/gbskernels_ext.cpp:209-228; tests/test_workspace.py for the model)."""

from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
RNG = np.random.default_rng(123)


def sym(N, scale=0.5):
    X = RNG.standard_normal((N, N)) + 1j * RNG.standard_normal((N, N))
    return scale * (X + X.T) / 2


def phys_O(n):
    X = RNG.standard_normal((2 * n, 2 * n))
    S = X @ X.T / (2 * n) + np.eye(2 * n)
    O = np.eye(2 * n) - np.linalg.inv(S)
    return (O + O.T) / 2


@pytest.mark.parametrize("func,make,d", [("perm", lambda: sym(9), 9), ("haf", lambda: sym(12), 12),
                                         ("lhaf", lambda: sym(11), 11), ("tor", lambda: phys_O(6), 12)])
@pytest.mark.parametrize("precision", ["fp64", "dd"])
def test_resident_equals_host(gpu, func, make, d, precision):
    mats = np.stack([make() for _ in range(5)])
    host = getattr(gpu, f"{func}_batched")(mats, precision=precision)
    with gpu.Workspace() as ws:
        r = getattr(ws, f"{func}_resident")(mats, precision=precision)
        assert np.array_equal(r.numpy(), host)
        assert np.array_equal(r.status.numpy(), np.zeros(5, np.int32))
        r.close()


def test_resident_certified_carries_the_bound(gpu):
    mats = np.stack([sym(10) for _ in range(4)])
    v, diags = gpu.haf_batched(mats, precision="certified", return_diagnostics=True)
    bounds = np.array([d["abs_error_bound"] for d in diags])
    with gpu.Workspace() as ws:
        r = ws.haf_resident(mats, precision="certified")
        assert np.array_equal(r.numpy(), v)
        assert np.array_equal(r.aux.numpy(), bounds)
        r.close()


def test_resident_auto_reruns_in_dd_on_device(gpu):
    # a cancelling permanent (kappa >= 1e8) next to a benign one
    from gbskernels_b200 import workloads
    bad = np.ones((12, 12), np.complex128)
    bad[0, :] = np.linspace(-1, 1, 12)
    bad[0, 0] += 1e-9
    good = np.stack(list(workloads.perm_haar_batch(1, 12, seed=5)))[0]
    mats = np.stack([good, bad])
    host, diags = gpu.perm_batched(mats, precision="auto", return_diagnostics=True)
    with gpu.Workspace() as ws:
        r = ws.perm_resident(mats, precision="auto")
        vals, kap = r.numpy(), r.aux.numpy()
        assert np.array_equal(vals, host)
        assert diags[1]["tier"] == "dd" and diags[0]["tier"] == "fp64"
        for i in range(2):
            assert kap[i] == pytest.approx(diags[i]["cancellation"], rel=1e-12)
        r.close()


def test_ragged_resident_in_request_order(gpu):
    funcs = ["haf", "perm", "tor", "lhaf", "haf", "haf", "perm"]
    mats = [sym(8), sym(6), phys_O(5), sym(7), np.zeros((0, 0)), sym(5), np.zeros((0, 0))]
    precs = ["fp64", "dd", "certified", "fp64", "fp64", "fp64", "certified"]
    with gpu.Workspace() as ws:
        host, st = ws.evaluate(funcs, mats, precs, return_status=True)
        r = ws.evaluate_resident(funcs, mats, precs)
        assert np.array_equal(r.numpy(), host)
        assert np.array_equal(r.status.numpy(), st)
        aux = r.aux.numpy()
        assert aux[4] == 1.0          # haf of the empty matrix: exact 1, indicator |1|
        assert aux[6] == 0.0          # certified exact value (perm of 0 x 0): bound 0
        assert aux[2] > 0.0           # certified torontonian: a positive bound
        r.close()


def test_resident_torch_zero_copy(gpu):
    import torch
    mats = np.stack([phys_O(5) for _ in range(3)])
    with gpu.Workspace() as ws:
        r = ws.tor_resident(mats, precision="certified")
        t = torch.as_tensor(r, device="cuda")
        b = torch.as_tensor(r.aux, device="cuda")
        s = torch.as_tensor(r.status, device="cuda")
        assert t.dtype == torch.complex128 and b.dtype == torch.float64 and s.dtype == torch.int32
        assert np.array_equal(t.cpu().numpy(), r.numpy())
        assert np.array_equal(b.cpu().numpy(), r.aux.numpy())
        assert int(s.abs().sum().item()) == 0
        del t, b, s
        r.close()


def test_resident_refusals(gpu):
    with gpu.Workspace() as ws:
        with pytest.raises(ValueError):
            ws.haf_resident([np.eye(4), np.eye(6)])
        with pytest.raises(NotImplementedError):
            ws.haf_resident(np.stack([np.eye(4)]), precision="ref")
        A = sym(6)
        A[0, 1] = np.inf
        with pytest.raises(ValueError):
            ws.haf_resident(A[None], precision="certified")


def test_resident_dlpack_export(gpu):
    # DLPack (the reference's resident contract): zero-copy tensors over the block;
    # close() while a tensor is alive is deferred until the tensor is released
    import gc

    import torch
    from gbskernels_b200 import _dlpack
    mats = np.stack([sym(10) for _ in range(4)])
    with gpu.Workspace() as ws:
        r = ws.haf_resident(mats, precision="certified")
        host, bnd = r.numpy(), r.aux.numpy()
        assert r.__dlpack_device__() == (2, torch.cuda.current_device())
        t = torch.from_dlpack(r)
        a = torch.from_dlpack(r.aux)
        st = torch.from_dlpack(r.status)
        assert t.dtype == torch.complex128 and a.dtype == torch.float64 and st.dtype == torch.int32
        assert t.data_ptr() == r.__cuda_array_interface__["data"][0]  # no copy
        assert np.array_equal(t.cpu().numpy(), host) and np.array_equal(a.cpu().numpy(), bnd)
        r.close()  # deferred: three tensors still reference the block
        assert r._ptr and np.array_equal(t.cpu().numpy(), host)
        del t, a, st
        gc.collect()
        assert not r._ptr and not _dlpack._LIVE  # released with the last tensor
