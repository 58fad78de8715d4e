"""Autotuner for the work-item split and the per-size block size.

    python -m gbskernels_b200.autotune --out tuned.json       # tune, apply, save
    gbskernels_b200.autotune.load("tuned.json")               # apply a saved table

For each (function, tier class, evaluated side) of a tuning set it times the
candidates on a synthetic batch of that size through a device-resident plan in
per-size mode (one launch per bucket, the session's CUDA-event kernel time of the
last of `reps` runs) and keeps the fastest:

  * split -- log2 of the work per item: haf / lhaf subsets per item, perm Gray steps
    per lane, tor prefix leaves per item (32 tail subsets each); more work per item
    means fewer items (less queue and reduction overhead) but coarser load balance;
  * warps -- warps per block of the per-size launches (1, 2 or 4), where the
    workspace allows more than one.

The choice is applied process-wide through ``gbs_set_split`` (the planner reads it
for every later plan, persistent or per-size) and saved as JSON keyed by the GPU
name.  The binary64 tiers (fp64, indicator, certified) share one entry, so their
values stay bit-identical after tuning; a tuned split changes the summation
grouping, so values can differ from the untuned ones in the last bits.
"""

from __future__ import annotations

import argparse
import json
from pathlib import Path

import numpy as np

from . import _lib, workloads
from .configs import run

_FN = {"perm": 0, "haf": 1, "lhaf": 2, "tor": 3}
# default tuning set: (function, evaluated side, split candidates)
DEFAULT_SET = (
    [("haf", N, (5, 6, 7, 8)) for N in (16, 20, 24, 28)]
    + [("lhaf", N, (5, 6, 7, 8)) for N in (16, 20, 24, 28)]
    + [("perm", n, (8, 9, 10, 11)) for n in (20, 24)]
    + [("tor", 2 * k, (7, 8, 9, 10)) for k in (16, 20, 24)]
)
WARPS = (1, 2, 4)


def _batch(func: str, dim: int, B: int, seed: int) -> list[np.ndarray]:
    rng = np.random.default_rng(seed)
    if func in ("haf", "lhaf"):
        A = workloads.gbs_kernel(100, 1.0, seed)
        out = []
        for _ in range(B):
            idx = np.sort(rng.integers(0, 100, size=dim))
            S = A[np.ix_(idx, idx)].copy()
            if func == "lhaf":
                S[np.diag_indices(dim)] = 0.3 * (rng.standard_normal(dim) + 1j * rng.standard_normal(dim))
            out.append(S)
        return out
    if func == "perm":
        return list(workloads.perm_haar_batch(B, dim, seed=seed))
    return list(workloads.tor_click_batch(B, kmin=dim // 2, kmax=dim // 2, seed=seed))


def _batch_size(func: str, dim: int) -> int:
    # about 10-50 ms of kernel time per candidate on one B200
    if func in ("haf", "lhaf"):
        return {16: 4096, 20: 2048, 24: 512, 28: 128}.get(dim, 256)
    if func == "perm":
        return {20: 1024, 24: 64}.get(dim, 64)
    return {32: 2048, 40: 256, 48: 16}.get(dim, 64)


def set_split(func: str, tier: str, dim: int, split: int, warps: int = 0) -> None:
    t = {"fp64": 0, "dd": 1, "kappa": 2, "certified": 3}[tier]
    _lib.check(_lib.load().gbs_set_split(_FN[func], t, dim, split, warps), "gbs_set_split")


def get_split(func: str, tier: str, dim: int) -> tuple[int, int]:
    t = {"fp64": 0, "dd": 1, "kappa": 2, "certified": 3}[tier]
    s = np.zeros(1, np.int32)
    w = np.zeros(1, np.int32)
    _lib.check(_lib.load().gbs_get_split(_FN[func], t, dim, _lib.iptr(s), _lib.iptr(w)), "gbs_get_split")
    return int(s[0]), int(w[0])


def clear() -> None:
    """Back to the planner's defaults for every entry."""
    for f in _FN:
        for tier in ("fp64", "dd"):
            for dim in range(65):
                set_split(f, tier, dim, -1, 0)


def _device_name() -> str:
    try:
        import torch
        return torch.cuda.get_device_name(0)
    except Exception:  # pragma: no cover
        return "cuda:0"


def tune(tuning_set=DEFAULT_SET, tier: str = "fp64", reps: int = 2, seed: int = 11, verbose: bool = False) -> dict:
    """Time every candidate, apply the best, return the table {key: {...}}."""
    table = {}
    for func, dim, splits in tuning_set:
        mats = _batch(func, dim, _batch_size(func, dim), seed)
        best = None
        trials = []
        for sp in splits:
            for w in WARPS:
                set_split(func, tier, dim, sp, w)
                res, *_ = run(func, mats, tier, per_size=True, reps=reps)
                trials.append((res["kernel_ms"], sp, w))
                if best is None or res["kernel_ms"] < best[0]:
                    best = (res["kernel_ms"], sp, w)
        set_split(func, tier, dim, best[1], best[2])
        key = f"{func}/{tier}/{dim}"
        table[key] = {"split": best[1], "warps": best[2], "kernel_ms": best[0],
                      "trials": [{"split": s, "warps": w, "kernel_ms": t} for t, s, w in trials]}
        if verbose:
            print(key, table[key]["split"], table[key]["warps"], f"{best[0]:.3f} ms", flush=True)
    return table


def save(table: dict, path: str | Path) -> None:
    p = Path(path)
    data = json.loads(p.read_text()) if p.exists() else {}
    data[_device_name()] = {k: {"split": v["split"], "warps": v["warps"], "kernel_ms": v["kernel_ms"],
                                "trials": v.get("trials", [])} for k, v in table.items()}
    p.write_text(json.dumps(data, indent=1))


def load(path: str | Path, device: str | None = None) -> int:
    """Apply a saved table for this GPU (or `device`); returns the entries applied."""
    data = json.loads(Path(path).read_text())
    entries = data.get(device or _device_name(), {})
    for key, v in entries.items():
        func, tier, dim = key.split("/")
        set_split(func, tier, int(dim), int(v["split"]), int(v["warps"]))
    return len(entries)


def main(argv=None) -> None:
    ap = argparse.ArgumentParser(description="tune work-item splits and block sizes on this GPU")
    ap.add_argument("--out", default=None, help="JSON file to save the table into (keyed by GPU name)")
    ap.add_argument("--reps", type=int, default=2)
    a = ap.parse_args(argv)
    table = tune(reps=a.reps, verbose=True)
    if a.out:
        save(table, a.out)


if __name__ == "__main__":
    main()
