"""Generate tests/golden/golden.npz from the REFERENCE implementation.

Run where a reference checkout is available, naming it with --ref (or the
GBS_REFERENCE_DIR environment variable):

    python tests/golden/make_golden.py --ref <reference tree>

For seeded small inputs of every function it records
  * the reference's mpmath ground truth (highprec_ref.*_mp, 40 digits) as (hi, lo)
    binary64 pairs,
  * the reference's binary64 CPU values (cpu_ref.perm / haf / lhaf / tor),
  * the reference's sum|term| cancellation indicators (cpu_ref diagnostics),
  * the reference's certified enclosures (cpu_ref.certified) -- value and bound.
The fixture is read by the tests on any machine; the reference itself is not needed
at test time.
"""

from __future__ import annotations

import argparse
import os
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent


def _mp_pair(x) -> tuple[float, float, float, float]:
    import mpmath
    with mpmath.workdps(40):
        z = mpmath.mpc(x)
        re_hi = float(z.real)
        re_lo = float(z.real - re_hi)
        im_hi = float(z.imag)
        im_lo = float(z.imag - im_hi)
    return re_hi, re_lo, im_hi, im_lo


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default=os.environ.get("GBS_REFERENCE_DIR"),
                    help="reference checkout (default: $GBS_REFERENCE_DIR)")
    ap.add_argument("--out", default=str(HERE / "golden.npz"))
    args = ap.parse_args()
    if not args.ref:
        ap.error("name the reference checkout with --ref or GBS_REFERENCE_DIR")
    sys.path.insert(0, args.ref)
    import cpu_ref  # noqa: E402  (reference package)
    import highprec_ref  # noqa: E402
    from cpu_ref import diagnostics  # noqa: E402

    rng = np.random.default_rng(20261203)
    cases: dict[str, list] = {f: [] for f in ("perm", "haf", "lhaf", "tor")}

    def sym(N, cplx=True, scale=1.0):
        X = rng.uniform(-1, 1, (N, N)) + (1j * rng.uniform(-1, 1, (N, N)) if cplx else 0)
        return scale * (X + X.T) / 2

    def phys_O(n):
        X = rng.standard_normal((2 * n, 2 * n))
        S = X @ X.T / (2 * n) + np.eye(2 * n)
        O = np.eye(2 * n) - np.linalg.inv(S)
        return (O + O.T) / 2

    for n in range(1, 9):
        for k in range(3):
            A = rng.uniform(-1, 1, (n, n)) + 1j * rng.uniform(-1, 1, (n, n))
            cases["perm"].append(A)
        cases["perm"].append(np.where(rng.random((n, n)) < 0.5, -1.0, 1.0).astype(np.complex128))
    for N in range(2, 11, 2):
        for k in range(3):
            cases["haf"].append(sym(N))
        cases["haf"].append(sym(N, cplx=False))
    for N in range(1, 10):
        for k in range(3):
            cases["lhaf"].append(sym(N))
    for n in range(1, 6):
        for k in range(3):
            cases["tor"].append(phys_O(n).astype(np.complex128))
        O = phys_O(n) * 0.5 + 1j * 0.05 * sym(2 * n, cplx=False)
        cases["tor"].append(O)  # complex O: per-subset LU path

    mp = {"perm": highprec_ref.permanent_mp, "haf": highprec_ref.hafnian_mp,
          "lhaf": highprec_ref.loop_hafnian_mp, "tor": highprec_ref.torontonian_mp}
    fp = {"perm": cpu_ref.perm, "haf": cpu_ref.haf, "lhaf": cpu_ref.lhaf, "tor": cpu_ref.tor}
    absfn = {"perm": diagnostics.glynn_abs_term_sum, "haf": diagnostics.hafnian_abs_term_sum,
             "lhaf": diagnostics.loop_hafnian_abs_term_sum, "tor": diagnostics.torontonian_abs_term_sum}
    out: dict[str, np.ndarray] = {}
    for f, mats in cases.items():
        dims = np.array([m.shape[0] for m in mats], dtype=np.int32)
        pad = max(int(dims.max()), 1)
        stack = np.zeros((len(mats), pad, pad), dtype=np.complex128)
        for i, m in enumerate(mats):
            stack[i, : m.shape[0], : m.shape[0]] = m
        mpv = np.array([_mp_pair(mp[f](m, dps=40)) for m in mats], dtype=np.float64)
        fpv = np.array([complex(fp[f](m)) for m in mats], dtype=np.complex128)
        def _abs(m):
            if f == "lhaf" and m.shape[0] % 2:
                # odd N: the indicator of the augmented A (+) [1] the GPU path evaluates
                a = np.zeros((m.shape[0] + 1,) * 2, dtype=np.complex128)
                a[:-1, :-1] = m
                a[-1, -1] = 1.0
                m = a
            return float(absfn[f](m))
        absn = np.array([_abs(m) for m in mats], dtype=np.float64)
        cv, cb = [], []
        for m in mats:
            try:
                v, b = cpu_ref.certified(f, m)
                cv.append(complex(v)); cb.append(float(b))
            except Exception:  # the reference refuses some inputs
                cv.append(complex(np.nan, np.nan)); cb.append(np.inf)
        out[f"{f}_dims"] = dims
        out[f"{f}_mats"] = stack
        out[f"{f}_mp"] = mpv
        out[f"{f}_cpu_fp64"] = fpv
        out[f"{f}_absnorm"] = absn
        out[f"{f}_cert_value"] = np.array(cv, dtype=np.complex128)
        out[f"{f}_cert_bound"] = np.array(cb, dtype=np.float64)
        print(f"{f}: {len(mats)} cases, max dim {pad}")
    np.savez_compressed(args.out, **out)
    print("wrote", args.out)


if __name__ == "__main__":
    main()
