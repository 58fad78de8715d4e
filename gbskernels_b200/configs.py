"""Runner for the synthetic workloads beside the headline mixed queue.

    python -m gbskernels_b200.configs haf16              # 4096 real symmetric 16x16 hafnians
    python -m gbskernels_b200.configs perm20 --tier dd   # 1024 Haar 20x20 permanents
    python -m gbskernels_b200.configs tor --tier certified              # 8192 click patterns, 10..24 modes
    python -m gbskernels_b200.configs tor --batch 64 --kmin 18 --kmax 20  # small case for ncu
    python -m gbskernels_b200.configs serve              # serving at 1e3 .. 1e5 requests/s

Each run uploads the batch once (a device-resident queue), evaluates it once to
warm up, then `--reps` more times; the kernel time is the session's own CUDA-event
time of the last evaluation.  One JSON line: instances/s over the kernel time, the
launch count, how many instances finished with status ok, and for the certified
tier the median and maximum relative bound.  `--mode per-size` uses one launch per
(function, tier, size) bucket instead of the persistent queue.

`serve` replays the chain-rule query stream (haf / lhaf / tor, N 6..30, fp64 70 % /
auto 20 % / certified 10 %) against the continuous-batching server at each Poisson
arrival rate of `--rates` (default 1e3, 3e3, 1e4, 3e4, 1e5 requests/s), one JSON
line per rate: throughput, p50 / p99 latency, and the offline rate of the same
requests as one batch (measured once).
"""

from __future__ import annotations

import argparse
import json

import numpy as np

from . import Workspace, _lib, _pack, workloads

_FN = {"perm": 0, "haf": 1, "lhaf": 2, "tor": 3}
_TIER = {"fp64": 0, "dd": 1, "kappa": 2, "certified": 3, "certified-dd": 4}


def run(func: str, mats: list, tier: str = "fp64", per_size: bool = False, reps: int = 1) -> dict:
    lib = _lib.load()
    B = len(mats)
    buf, dims, offs = _pack(mats)
    fc = np.full(B, _FN[func], np.int32)
    ti = np.full(B, _TIER[tier], np.int32)
    out = np.empty(B, np.complex128)
    aux = np.empty(B)
    st = np.zeros(B, np.int32)
    with Workspace() as ws:
        s = ws._session
        _lib.check(lib.gbs_queue_prepare(s, B, _lib.iptr(fc), _lib.iptr(ti), _lib.iptr(dims), _lib.llptr(offs),
                                         _lib.dptr(buf.view(np.float64)), 1 if per_size else 0), "gbs_queue_prepare")
        for _ in range(1 + max(reps, 1)):
            _lib.check(lib.gbs_queue_run(s, None), "gbs_queue_run")
            _lib.check(lib.gbs_queue_read(s, None, _lib.dptr(out.view(np.float64)), _lib.dptr(aux),
                                          _lib.iptr(st)), "gbs_queue_read")
        stats = ws.last_stats()
    res = {"func": func, "tier": tier, "batch": B, "mode": "per-size" if per_size else "persistent",
           "kernel_ms": stats["kernel_ms"], "instances_per_s": B / stats["kernel_ms"] * 1e3,
           "launches": stats["launches"], "items": stats["items"], "status_ok": int((st == 0).sum())}
    if tier in ("certified", "certified-dd"):
        rel = aux / np.maximum(np.abs(out), 1e-300)
        res["rel_bound_median"] = float(np.median(rel))
        res["rel_bound_max"] = float(np.max(rel))
    return res, out, aux, st


def main(argv=None) -> None:
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("workload", choices=["haf16", "perm20", "tor", "serve"])
    ap.add_argument("--tier", default="fp64", choices=list(_TIER))
    ap.add_argument("--batch", type=int, default=None)
    ap.add_argument("--kmin", type=int, default=10)
    ap.add_argument("--kmax", type=int, default=24)
    ap.add_argument("--seed", type=int, default=None)
    ap.add_argument("--mode", default="persistent", choices=["persistent", "per-size"])
    ap.add_argument("--reps", type=int, default=1)
    ap.add_argument("--rates", default="1e3,3e3,1e4,3e4,1e5")
    ap.add_argument("--requests", type=int, default=2000)
    a = ap.parse_args(argv)
    if a.workload == "serve":
        from .serving import offline_rate, serve_stream

        seed = 5 if a.seed is None else a.seed
        off = offline_rate(a.requests, seed)
        for r in (float(x) for x in a.rates.split(",")):
            res = serve_stream(rate=r, n_req=a.requests, seed=seed, offline=off)
            print(json.dumps(res), flush=True)
        return
    if a.workload == "haf16":
        mats = list(workloads.haf_real_batch(a.batch or 4096, 16, seed=1 if a.seed is None else a.seed))
        func = "haf"
    elif a.workload == "perm20":
        mats = list(workloads.perm_haar_batch(a.batch or 1024, 20, seed=2 if a.seed is None else a.seed))
        func = "perm"
    else:
        mats = list(workloads.tor_click_batch(a.batch or 8192, kmin=a.kmin, kmax=a.kmax,
                                              seed=4 if a.seed is None else a.seed))
        func = "tor"
    res, *_ = run(func, mats, a.tier, a.mode == "per-size", a.reps)
    print(json.dumps(res), flush=True)


if __name__ == "__main__":
    main()
