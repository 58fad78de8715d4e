// perm_tor.cuh -- permanent (Glynn / Gray code) work-item evaluators, binary64 and
// double-double.  (The torontonian walks live in tor_warp.cuh / tor_warp_dd.cuh.)
//
// Permanent (reference: cpu_ref/permanent.py:108-139, core/permanent.cu:30-76):
//   perm(A) = 2^-(n-1) sum_{delta, delta_0 = +1} (prod delta) prod_r sum_c delta_c A[r][c],
//   delta walked in Gray order: step i flips column ctz(i)+1, a +-2 A[:, col] update
//   of the row-sum vector.  B200 mapping: a work item is a power-of-two aligned range
//   of Gray indices split evenly over the 32 lanes; every lane keeps its own row-sum
//   vector in registers (the matrix side n is a template parameter) and, because the
//   lane ranges are aligned, all lanes flip the same column at the same step, so the
//   column reads from shared memory are warp broadcasts.  The row product is a
//   balanced tree.  Lane partials are combined in a fixed shuffle tree.
#pragma once

#include "gbs_common.cuh"

namespace gbsb {

constexpr int kPermMaxN = 32;

// ----------------------------------------------------------------- permanent, binary64
// Balanced product tree over an array of NN complex values (NN compile-time).
template <int NN>
__device__ __forceinline__ cplx tree_prod(const cplx (&v)[NN]) {
  if constexpr (NN == 1) {
    return v[0];
  } else {
    constexpr int H = NN / 2;
    cplx lo[H], hi[NN - H];
#pragma unroll
    for (int i = 0; i < H; ++i) lo[i] = v[i];
#pragma unroll
    for (int i = 0; i < NN - H; ++i) hi[i] = v[H + i];
    return cmul(tree_prod<H>(lo), tree_prod<NN - H>(hi));
  }
}

// Sum of the signed Glynn terms over Gray indices [i0, i0 + R) for one lane, where
// R is a power of two and i0 a multiple of R.  A2 = 2*A staged in shared memory
// (row-major complex).  Returns sum and (optionally) sum |term|.
template <int NN, bool KAPPA>
__device__ __forceinline__ cplx perm_lane_range(const double* __restrict__ A2, uint64_t i0, uint64_t R,
                                                double& absacc) {
  cplx rs[NN];
  const uint64_t g0 = gray_of(i0);
  // row sums at delta(i0): delta_0 = +1, delta_{c+1} = -1 iff bit c of gray(i0)
#pragma unroll
  for (int r = 0; r < NN; ++r) {
    cplx s = mkc(0.0, 0.0);
#pragma unroll 4
    for (int c = 0; c < NN; ++c) {
      cplx a = ld_c2(A2 + (r * NN + c) * 2);
      double sg = (c > 0 && ((g0 >> (c - 1)) & 1ull)) ? -0.5 : 0.5;  // A2 holds 2A
      s.re = fma(sg, a.re, s.re);
      s.im = fma(sg, a.im, s.im);
    }
    rs[r] = s;
  }
  cplx acc = mkc(0.0, 0.0);
  double sign = (i0 & 1ull) ? -1.0 : 1.0;
  {
    cplx p = tree_prod<NN>(rs);
    acc = cplx{sign * p.re, sign * p.im};
    if (KAPPA) absacc += cabs_fast(p);
  }
  for (uint64_t j = 1; j < R; ++j) {
    const uint64_t i = i0 + j;
    const int k = __ffsll((long long)j) - 1;  // == ctz(i) since i0 is a multiple of R > j
    const double step = ((gray_of(i) >> k) & 1ull) ? -1.0 : 1.0;
    const double* col = A2 + (k + 1) * 2;
#pragma unroll
    for (int r = 0; r < NN; ++r) {
      cplx a = ld_c2(col + r * NN * 2);
      rs[r].re = fma(step, a.re, rs[r].re);
      rs[r].im = fma(step, a.im, rs[r].im);
    }
    sign = -sign;
    cplx p = tree_prod<NN>(rs);
    acc.re = fma(sign, p.re, acc.re);
    acc.im = fma(sign, p.im, acc.im);
    if (KAPPA) absacc += cabs_fast(p);
  }
  return acc;
}

// ----------------------------------------------------------------- permanent, double-double
template <int NN>
__device__ __forceinline__ ddc tree_prod_dd(const ddc (&v)[NN]) {
  if constexpr (NN == 1) {
    return v[0];
  } else {
    constexpr int H = NN / 2;
    ddc lo[H], hi[NN - H];
#pragma unroll
    for (int i = 0; i < H; ++i) lo[i] = v[i];
#pragma unroll
    for (int i = 0; i < NN - H; ++i) hi[i] = v[H + i];
    return ddc_mul(tree_prod_dd<H>(lo), tree_prod_dd<NN - H>(hi));
  }
}

template <int NN>
__device__ __forceinline__ ddc perm_lane_range_dd(const double* __restrict__ A2, uint64_t i0, uint64_t R) {
  ddc rs[NN];
  const uint64_t g0 = gray_of(i0);
#pragma unroll
  for (int r = 0; r < NN; ++r) {
    ddc s = ddc{dd_make(0.0), dd_make(0.0)};
    for (int c = 0; c < NN; ++c) {
      cplx a = ld_c2(A2 + (r * NN + c) * 2);
      double sg = (c > 0 && ((g0 >> (c - 1)) & 1ull)) ? -0.5 : 0.5;  // exact scaling of 2A
      s = ddc{dd_add_d(s.re, sg * a.re), dd_add_d(s.im, sg * a.im)};
    }
    rs[r] = s;
  }
  ddc acc = ddc{dd_make(0.0), dd_make(0.0)};
  bool neg = (i0 & 1ull) != 0;
  {
    ddc p = tree_prod_dd<NN>(rs);
    acc = neg ? ddc_neg(p) : p;
  }
  for (uint64_t j = 1; j < R; ++j) {
    const uint64_t i = i0 + j;
    const int k = __ffsll((long long)j) - 1;
    const bool minus = ((gray_of(i) >> k) & 1ull) != 0;
    const double* col = A2 + (k + 1) * 2;
#pragma unroll
    for (int r = 0; r < NN; ++r) {
      cplx a = ld_c2(col + r * NN * 2);  // exact 2A
      rs[r].re = dd_add_d(rs[r].re, minus ? -a.re : a.re);
      rs[r].im = dd_add_d(rs[r].im, minus ? -a.im : a.im);
    }
    neg = !neg;
    ddc p = tree_prod_dd<NN>(rs);
    acc = neg ? ddc_sub(acc, p) : ddc_add(acc, p);
  }
  return acc;
}

}  // namespace gbsb
