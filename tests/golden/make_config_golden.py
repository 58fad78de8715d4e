"""Generate tests/golden/config_sizes.npz: truths at the benchmark configurations'
own sizes, for the GPU parity tests (test infrastructure).

    python tests/golden/make_config_golden.py [--jobs 8]

Inputs come from the seeded workload generators (gbskernels_b200.workloads) and
are stored in the fixture, so the tests do not depend on the generators staying
the same.  Truths:

  * config 1 (real symmetric 16 x 16 hafnians), config 2 (Haar 20 x 20
    permanents) and config 3 (hafnians and loop hafnians of photon-pattern
    submatrices, N = 22, 24, 26, 28): the binary128 oracle (oracle/gbs_oracle.cpp
    in __float128), stored as (hi, lo) pairs, plus the binary64 oracle's
    sum |term| (the cancellation indicator of the power trace / Glynn walk);
  * config 4 (threshold-detector torontonians, 18, 20, 22 and 24 modes): the
    binary128 oracle (recursive Cholesky) and the reference's own certified
    double-double single-large torontonian (core/tor_recursive.cu:523-678 through
    gbs_tor_single_ddcertified_host, compiled on the host into oracle/_ref by
    oracle/Makefile): value and rigorous radius.

The reference build is needed only here (it is absent where the tests run).
Runtime: about 15 minutes on 8 cores (the 24-mode torontonians dominate).
"""

from __future__ import annotations

import argparse
import multiprocessing as mp
import os
import sys
import time
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parents[1]


def _task(job):
    sys.path.insert(0, str(ROOT))
    import oracle
    kind, key, mat = job
    t0 = time.time()
    if kind in ("haf", "lhaf", "perm"):
        q = getattr(oracle, kind)(mat, "quad", hilo=True)
        _, absn = getattr(oracle, kind)(mat, "fp64", with_absnorm=True)
        res = {"quad": np.array(q), "absnorm": absn}
    elif kind == "tor_quad":
        q = oracle.tor(mat, "quad", hilo=True)
        _, absn = oracle.tor(mat, "fp64", with_absnorm=True)
        res = {"quad": np.array(q), "absnorm": absn}
    elif kind == "tor_ref":
        v, e = oracle.ref_tor_single_ddcertified(mat, 0)
        res = {"ref_value": v, "ref_bound": e}
    else:
        raise ValueError(kind)
    res["seconds"] = time.time() - t0
    return kind, key, res


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--jobs", type=int, default=len(os.sched_getaffinity(0)))
    ap.add_argument("--out", default=str(HERE / "config_sizes.npz"))
    args = ap.parse_args()
    sys.path.insert(0, str(ROOT))
    import oracle
    from gbskernels_b200 import workloads

    if not oracle.ref_available():
        raise SystemExit("oracle/_ref/libgbsref.so is missing: build it with the reference tree present")

    # ---- inputs
    c1 = workloads.haf_real_batch(8, 16, seed=1)
    c2 = workloads.perm_haar_batch(4, 20, seed=2)
    funcs, mats = workloads.mixed_haf_lhaf(3000, seed=3)
    c3 = []  # (func, matrix): 2 haf + 2 lhaf per size, first seen in generator order
    for N in (22, 24, 26, 28):
        for f in ("haf", "lhaf"):
            c3 += [(f, m) for g, m in zip(funcs, mats) if g == f and m.shape[0] == N][:2]
    tors = workloads.tor_click_batch(400, seed=4)
    c4 = []
    for k in (18, 20, 22, 24):
        c4 += [m for m in tors if m.shape[0] == 2 * k][:2]

    jobs = [("haf", ("c1", i), np.asarray(m, np.complex128)) for i, m in enumerate(c1)]
    jobs += [("perm", ("c2", i), m) for i, m in enumerate(c2)]
    jobs += [(f, ("c3", i), m) for i, (f, m) in enumerate(c3)]
    jobs += [("tor_quad", ("c4", i), m) for i, m in enumerate(c4)]
    jobs += [("tor_ref", ("c4", i), m) for i, m in enumerate(c4)]
    # longest first
    cost = {"haf": 1, "lhaf": 1, "perm": 1, "tor_quad": 2, "tor_ref": 3}
    jobs.sort(key=lambda j: -(j[2].shape[0] ** 2) * cost[j[0]])
    t0 = time.time()
    with mp.get_context("spawn").Pool(args.jobs) as pool:
        results = pool.map(_task, jobs, chunksize=1)
    print(f"[golden] {len(jobs)} jobs in {time.time() - t0:.0f} s", flush=True)
    R = {(k, key): r for k, key, r in results}

    out = {}
    out["c1_mats"] = np.stack(c1)
    out["c1_quad"] = np.stack([R[("haf", ("c1", i))]["quad"] for i in range(len(c1))])
    out["c1_absnorm"] = np.array([R[("haf", ("c1", i))]["absnorm"] for i in range(len(c1))])
    out["c2_mats"] = np.stack(c2)
    out["c2_quad"] = np.stack([R[("perm", ("c2", i))]["quad"] for i in range(len(c2))])
    out["c2_absnorm"] = np.array([R[("perm", ("c2", i))]["absnorm"] for i in range(len(c2))])
    n3 = len(c3)
    out["c3_funcs"] = np.array([f for f, _ in c3])
    out["c3_dims"] = np.array([m.shape[0] for _, m in c3], np.int32)
    pad = np.zeros((n3, 28, 28), np.complex128)
    for i, (_, m) in enumerate(c3):
        pad[i, :m.shape[0], :m.shape[0]] = m
    out["c3_mats"] = pad
    out["c3_quad"] = np.stack([R[(f, ("c3", i))]["quad"] for i, (f, _) in enumerate(c3)])
    out["c3_absnorm"] = np.array([R[(f, ("c3", i))]["absnorm"] for i, (f, _) in enumerate(c3)])
    n4 = len(c4)
    out["c4_dims"] = np.array([m.shape[0] for m in c4], np.int32)
    pad = np.zeros((n4, 48, 48), np.float64)
    for i, m in enumerate(c4):
        pad[i, :m.shape[0], :m.shape[0]] = m
    out["c4_mats"] = pad
    out["c4_quad"] = np.stack([R[("tor_quad", ("c4", i))]["quad"] for i in range(n4)])
    out["c4_absnorm"] = np.array([R[("tor_quad", ("c4", i))]["absnorm"] for i in range(n4)])
    out["c4_ref_value"] = np.array([R[("tor_ref", ("c4", i))]["ref_value"] for i in range(n4)])
    out["c4_ref_bound"] = np.array([R[("tor_ref", ("c4", i))]["ref_bound"] for i in range(n4)])
    out["generator"] = np.array("haf_real_batch(8,16,seed=1); perm_haar_batch(4,20,seed=2); "
                                "mixed_haf_lhaf(3000,seed=3) first 2 haf + 2 lhaf per N in 22..28; "
                                "tor_click_batch(400,seed=4) first 2 per k in 18..24")
    np.savez_compressed(args.out, **out)
    print(f"[golden] wrote {args.out}", flush=True)


if __name__ == "__main__":
    main()
