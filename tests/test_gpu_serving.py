"""Serving loop: continuous batching returns, for every request, the value the
same request gets alone (bit for bit for fp64 / certified), with resident states
gathered on the device, auto-tier escalation in the loop, and bounded latency."""

from __future__ import annotations

import numpy as np
import pytest

from gbskernels_b200 import workloads

pytestmark = pytest.mark.gpu


def test_served_equals_alone_bitwise(gpu):
    reqs = workloads.serving_stream(300, rate=1e5, seed=11, nmax=20)
    with gpu.Server(slots=3, budget_bytes=1 << 17) as srv:
        tickets = [srv.submit(f, m, p) for _, f, p, m in reqs]
        served = [srv.result(t) for t in tickets]
        st = srv.stats()
    assert st["batches"] > 3  # the stream was split over several overlapping batches
    with gpu.Workspace() as ws:
        for (_, f, p, m), (v, info) in zip(reqs, served):
            if p == "fp64":
                alone = ws.evaluate([f], [m], ["fp64"])[0]
                assert v == alone
            elif p == "certified":
                alone = ws.evaluate([f], [m], ["certified"])[0]
                assert v == alone or (np.isnan(v) and np.isnan(alone))
                assert info["tier"] == "certified-fp64"
            else:
                assert info["tier"] in ("fp64", "dd")
            assert info["latency_s"] >= 0


def test_resident_state_gather(gpu):
    M = 40
    A = workloads.gbs_kernel(M, 1.0, seed=2)
    rng = np.random.default_rng(3)
    gamma = (rng.standard_normal(M) + 1j * rng.standard_normal(M)) * 0.2
    with gpu.Server(slots=2) as srv:
        sid = srv.add_state(A, gamma)
        cases = []
        for N in (6, 9, 12, 16):
            idx = np.sort(rng.integers(0, M, size=N))
            sub = A[np.ix_(idx, idx)].copy()
            t1 = srv.submit_state("haf", sid, idx)
            subl = sub.copy()
            np.fill_diagonal(subl, gamma[idx])
            t2 = srv.submit_state("lhaf", sid, idx, use_gamma=True)
            cases.append((t1, "haf", sub))
            cases.append((t2, "lhaf", subl))
        for t, f, m in cases:
            v, _ = srv.result(t)
            assert v == getattr(gpu, f)(m), (f, m.shape)


def test_auto_escalates_inside_the_loop(gpu):
    # haf = delta * haf(R): three O(1) matchings cancel (kappa >> 1e8)
    g = np.random.default_rng(5)
    delta = 1e-10
    Bk = np.array([[0, 1, 1, 1], [1, 0, delta - 2, 1], [1, delta - 2, 0, 1], [1, 1, 1, 0]], dtype=complex)
    G2 = g.standard_normal((4, 4))
    R = G2 + G2.T
    np.fill_diagonal(R, 0)
    A = np.zeros((8, 8), dtype=complex)
    A[:4, :4], A[4:, 4:] = Bk, R
    with gpu.Server(slots=2) as srv:
        v, info = srv.result(srv.submit("haf", A, "auto"))
    assert info["tier"] == "dd"
    assert v == gpu.haf(A, precision="dd")


def test_server_rejects_bad_requests(gpu):
    with gpu.Server(slots=1) as srv:
        with pytest.raises(RuntimeError):
            srv.submit_state("haf", 7, [0, 1])
        sid = srv.add_state(np.eye(4))
        with pytest.raises(RuntimeError):
            srv.submit_state("haf", sid, [0, 9])
        with pytest.raises(RuntimeError):
            srv.submit_state("lhaf", sid, [0, 1], use_gamma=True)  # no loop weights uploaded


def test_chain_rule_stream_from_resident_states(gpu):
    """The serving benchmark's path: chain-rule queries (growing prefixes) on two
    resident states, gathered on the device, values bit-identical to the offline
    batch of host-gathered matrices, at a rate that keeps several batches in flight."""
    from gbskernels_b200.serving import serve_stream
    res = serve_stream(rate=2e4, n_req=400, seed=13, slots=3)
    assert res["values_equal_to_offline_batch"], res
    assert res["path"].startswith("resident")
    assert res["batches"] > 3 and res["p99_ms"] >= res["p50_ms"] > 0
