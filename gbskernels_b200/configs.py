"""Runner for the synthetic workloads beside the headline mixed queue.

    python -m gbskernels_b200.configs haf16              # 4096 real symmetric 16x16 hafnians
    python -m gbskernels_b200.configs perm20 --tier dd   # 1024 Haar 20x20 permanents
    python -m gbskernels_b200.configs tor --tier certified              # 8192 click patterns, 10..24 modes
    python -m gbskernels_b200.configs tor --batch 64 --kmin 18 --kmax 20  # small case for ncu
    python -m gbskernels_b200.configs serve              # serving at 1e3 .. 1e5 requests/s
    python -m gbskernels_b200.configs sieve              # 4096 repeated-row loop hafnians (M = 12)
    python -m gbskernels_b200.configs sampler            # 100,000 resident-chain samples (M 8 / 4)

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


def sieve_rate(n_patterns: int = 4096, M: int = 12, nmax: int = 3, seed: int = 6) -> dict:
    """Repeated-row loop hafnians (the finite-difference sieve, lhaf_repeated): random
    repetition patterns n_i in 0..nmax over an M-mode kernel A = U diag(tanh 1) U^T
    with loop weights gamma ~ CN(0, 0.1); fp64 and certified, each the median of 3
    host calls (allocation and copies included) after the same call once to warm up."""
    from . import lhaf_repeated
    rng = np.random.default_rng(seed)
    A = workloads.gbs_kernel(M, 1.0, seed)
    g = np.sqrt(0.05) * (rng.standard_normal(M) + 1j * rng.standard_normal(M))
    reps = rng.integers(0, nmax + 1, size=(n_patterns, M)).astype(np.int32)
    terms = float(np.prod(reps.astype(np.float64) + 1.0, axis=1).sum())
    t, v = _median_call(lambda: lhaf_repeated(A, g, reps))
    tc, (vc, diag) = _median_call(lambda: lhaf_repeated(A, g, reps, certified=True))
    rel = np.asarray(diag["abs_error_bound"]) / np.maximum(np.abs(vc), 1e-300)
    return {"patterns": n_patterns, "M": M, "nmax": nmax, "terms": terms,
            "patterns_per_s": n_patterns / t, "terms_per_s": terms / t,
            "certified_patterns_per_s": n_patterns / tc, "certified_rel_bound_median": float(np.median(rel)),
            "certified_values_equal_fp64": bool(np.array_equal(v, vc))}


def _median_call(fn, reps: int = 3):
    """(median seconds of `reps` calls after one warm-up call, the last result)."""
    import time
    fn()
    ts, r = [], None
    for _ in range(reps):
        t0 = time.perf_counter()
        r = fn()
        ts.append(time.perf_counter() - t0)
    return float(np.median(ts)), r


def sampler_rate(num_samples: int = 100000, cases=((8, 2), (4, 4)), seed: int = 7) -> list:
    """The resident sampler chain (gbs_sampler_sample): num_samples draws of M modes
    at photon cutoff c from a lossy squeezed state, the median of 3 host calls (the
    reduced matrices uploaded inside each) after the same call once to warm up."""
    from .sampler import sample_resident
    out = []
    for M, cutoff in cases:
        cov = workloads.lossy_squeezed_cov(M, seed=seed)
        t, s = _median_call(lambda: sample_resident(cov, num_samples, cutoff=cutoff, seed=2))
        out.append({"M": M, "cutoff": cutoff, "samples": num_samples, "samples_per_s": num_samples / t,
                    "mean_photons": float(s.sum(axis=1).mean())})
    return out


def main(argv=None) -> None:
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("workload", choices=["haf16", "perm20", "tor", "serve", "sieve", "sampler"])
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
    if a.workload == "sieve":
        print(json.dumps(sieve_rate()), flush=True)
        return
    if a.workload == "sampler":
        for r in sampler_rate():
            print(json.dumps(r), flush=True)
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
