"""Autotuner: tuning a small set applies a split from the candidates, values stay
correct and the binary64 tiers stay bit-identical under the tuned split; clearing
restores the planner's defaults.  Also the captured launch graph of a re-run plan
gives the same values as direct launches."""

from __future__ import annotations

import numpy as np
import pytest

from conftest import rel_err

pytestmark = pytest.mark.gpu


def test_tune_apply_and_clear(gpu, orc):
    from gbskernels_b200 import autotune, workloads
    try:
        table = autotune.tune([("haf", 16, (5, 7)), ("tor", 28, (7, 9))], reps=1)
        assert autotune.get_split("haf", "fp64", 16) == (table["haf/fp64/16"]["split"], table["haf/fp64/16"]["warps"])
        assert table["haf/fp64/16"]["split"] in (5, 7) and table["tor/fp64/28"]["split"] in (7, 9)
        mats = np.stack(list(workloads.haf_real_batch(6, 16, seed=3)))
        v = gpu.haf_batched(mats)
        for i in range(3):
            assert rel_err(v[i], orc.haf(mats[i], "quad")) < 1e-12
        O = np.stack(list(workloads.tor_click_batch(4, kmin=14, kmax=14, seed=5)))
        f = gpu.tor_batched(O)
        c, _ = gpu.tor_batched(O, precision="certified", return_diagnostics=True)
        assert np.array_equal(f, c)
        # a forced split changes the grouping, not the value beyond rounding
        autotune.set_split("tor", "fp64", 28, 6, 0)
        f2 = gpu.tor_batched(O)
        _, d = gpu.tor_batched(O, precision="auto", return_diagnostics=True)
        for i in range(4):
            assert rel_err(f2[i], f[i]) < max(1e-13, 1e-14 * d[i]["cancellation"]), i
    finally:
        autotune.clear()
    assert autotune.get_split("haf", "fp64", 16) == (-1, 0)


def test_graph_replay_equals_direct_launch(gpu):
    import ctypes
    from gbskernels_b200 import _lib, _pack, workloads
    lib = _lib.load()
    funcs = ["haf", "lhaf", "tor", "haf"]
    mats = [workloads.haf_real_batch(1, 12, seed=1)[0].astype(np.complex128),
            workloads.haf_real_batch(1, 10, seed=2)[0].astype(np.complex128),
            workloads.tor_click_batch(1, kmin=12, kmax=12, seed=3)[0],
            workloads.haf_real_batch(1, 16, seed=4)[0].astype(np.complex128)]
    buf, dims, offs = _pack(mats)
    fc = np.array([{"haf": 1, "lhaf": 2, "tor": 3}[f] for f in funcs], np.int32)
    ti = np.zeros(4, np.int32)
    outs = {}
    for graphs in (0, 1):
        with gpu.Workspace() as ws:
            s = ws._session
            _lib.check(lib.gbs_session_set_graphs(s, graphs), "set_graphs")
            for mode in (0, 1):
                _lib.check(lib.gbs_queue_prepare(s, 4, _lib.iptr(fc), _lib.iptr(ti), _lib.iptr(dims),
                                                 _lib.llptr(offs), _lib.dptr(buf.view(np.float64)), mode), "prep")
                for run in range(3):  # run 2 captures the graph, run 3 replays it
                    _lib.check(lib.gbs_queue_run(s, None), "run")
                    out = np.empty(4, np.complex128)
                    _lib.check(lib.gbs_queue_read(s, None, _lib.dptr(out.view(np.float64)), None, None), "read")
                    outs[(graphs, mode, run)] = out
    ref = outs[(0, 0, 0)]
    for k, v in outs.items():
        assert np.array_equal(v, ref), k
