"""Generate tests/golden/golden_repeated.npz from the REFERENCE implementation.

    python tests/golden/make_golden_repeated.py --ref <reference tree>   (or GBS_REFERENCE_DIR)

Seeded repeated-row loop-hafnian cases (base matrix A, loop weights gamma, one
repetition pattern each; small enough that the expansion's mpmath value is cheap):
  * the reference's finite-difference sieve in binary64 (cpu_ref.lhaf_repeated),
  * the reference's 40-digit mpmath loop hafnian of the EXPANDED matrix
    (highprec_ref.loop_hafnian_mp; the diagonal of copy i carries gamma_i), as
    (re_hi, re_lo, im_hi, im_lo).
"""

from __future__ import annotations

import argparse
import os
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default=os.environ.get("GBS_REFERENCE_DIR"),
                    help="reference checkout (default: $GBS_REFERENCE_DIR)")
    ap.add_argument("--out", default=str(HERE / "golden_repeated.npz"))
    args = ap.parse_args()
    if not args.ref:
        ap.error("name the reference checkout with --ref or GBS_REFERENCE_DIR")
    sys.path.insert(0, args.ref)
    import mpmath
    import cpu_ref  # noqa: E402  (reference package)
    import highprec_ref  # noqa: E402

    rng = np.random.default_rng(20261204)
    Mmax = 6
    As, gs, reps, sieve, mp = [], [], [], [], []
    for M in range(1, Mmax + 1):
        for k in range(4):
            X = rng.uniform(-1, 1, (M, M)) + 1j * rng.uniform(-1, 1, (M, M))
            A = (X + X.T) / 2
            g = (rng.uniform(-1, 1, M) + 1j * rng.uniform(-1, 1, M)) * (0.0 if k == 0 else 0.5)
            while True:
                r = rng.integers(0, 4, M)
                if 0 < r.sum() <= 10:
                    break
            idx = np.repeat(np.arange(M), r)
            E = A[np.ix_(idx, idx)].copy()
            np.fill_diagonal(E, g[idx])
            v = highprec_ref.loop_hafnian_mp(E, dps=40)
            with mpmath.workdps(40):
                z = mpmath.mpc(v)
                pair = (float(z.real), float(z.real - float(z.real)), float(z.imag), float(z.imag - float(z.imag)))
            Ap = np.zeros((Mmax, Mmax), np.complex128)
            Ap[:M, :M] = A
            gp = np.zeros(Mmax, np.complex128)
            gp[:M] = g
            rp = np.zeros(Mmax, np.int32)
            rp[:M] = r
            As.append(Ap)
            gs.append(gp)
            reps.append(rp)
            sieve.append(complex(cpu_ref.lhaf_repeated(A, g, r)))
            mp.append(pair)
    np.savez_compressed(args.out, A=np.array(As), gamma=np.array(gs), reps=np.array(reps),
                        M=np.repeat(np.arange(1, Mmax + 1), 4).astype(np.int32),
                        cpu_sieve=np.array(sieve), mp=np.array(mp))
    print(f"wrote {args.out}: {len(As)} cases")


if __name__ == "__main__":
    main()
