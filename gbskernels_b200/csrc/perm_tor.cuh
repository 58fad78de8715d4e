// perm_tor.cuh -- permanent (Glynn / Gray code) and torontonian (recursive prefix
// Cholesky) work-item evaluators, binary64 and double-double.
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
//
// Torontonian (reference: core/tor_recursive.cu:41-115, cpu_ref/tor_recursive.py:46-100):
//   tor(O) = sum_{S subset modes} (-1)^(n-|S|) / sqrt(det(I - O_S)), xxpp ordering,
//   det by a prefix Cholesky factor: including mode j appends its x- and p-rows
//   (O(|S|^2)), det(I - O_S) = prod (l_xx l_pp)^2.  B200 mapping: a work item fixes
//   the include pattern of the first g modes for each lane (32 prefix patterns per
//   item); each lane enumerates the 2^(n-g) subsets of the remaining modes by a
//   binary counter whose lowest bit is the LAST mode, so every counter step
//   truncates the factor to the untouched prefix and appends exactly one mode
//   (the same amortised cost as the reference's depth-first walk, no stack).
#pragma once

#include "gbs_common.cuh"

namespace gbsb {

constexpr int kPermMaxN = 32;
constexpr int kTorMaxModes = 32;           // dim 64 (single-large cap of the reference)
constexpr int kTorMaxDim = 2 * kTorMaxModes;

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

// ----------------------------------------------------------------- torontonian, binary64
// Append mode j's x- and p-rows to the packed lower-triangular factor L (row r at
// r(r+1)/2) for `count` already-included modes listed in modes[].  Returns false if
// I - O_S is not positive definite (off the physical domain).  detf = (l_xx l_pp)^2.
template <class T>
struct TorOps;

template <>
struct TorOps<double> {
  using V = double;
  __device__ static V zero() { return 0.0; }
  __device__ static V from(double x) { return x; }
  __device__ static V sub(V a, V b) { return a - b; }
  __device__ static V fms(V s, V a, V b) { return fma(-a, b, s); }
  __device__ static V div(V a, V b) { return a / b; }
  __device__ static V mul(V a, V b) { return a * b; }
  __device__ static V sqrt_(V a) { return sqrt(a); }
  __device__ static bool pos(V a) { return a > 0.0; }
  __device__ static double to_d(V a) { return a; }
  __device__ static V rsqrt_term(V det) { return 1.0 / sqrt(det); }
  __device__ static V add(V a, V b) { return a + b; }
  __device__ static V neg(V a) { return -a; }
};

template <>
struct TorOps<dd> {
  using V = dd;
  __device__ static V zero() { return dd_make(0.0); }
  __device__ static V from(double x) { return dd_make(x); }
  __device__ static V sub(V a, V b) { return dd_sub(a, b); }
  __device__ static V fms(V s, V a, V b) { return dd_sub(s, dd_mul(a, b)); }
  __device__ static V div(V a, V b) { return dd_div(a, b); }
  __device__ static V mul(V a, V b) { return dd_mul(a, b); }
  __device__ static V sqrt_(V a) { return dd_sqrt(a); }
  __device__ static bool pos(V a) { return a.hi > 0.0; }
  __device__ static double to_d(V a) { return a.hi + a.lo; }
  __device__ static V rsqrt_term(V det) { return dd_div(dd_make(1.0), dd_sqrt(det)); }
  __device__ static V add(V a, V b) { return dd_add(a, b); }
  __device__ static V neg(V a) { return dd_neg(a); }
};

template <class T>
__device__ __forceinline__ bool tor_append(const double* __restrict__ O, int n, int j, int count,
                                           const int* modes, T* L, T& detf) {
  using Op = TorOps<T>;
  const int dim = 2 * n;
  const int size = 2 * count;
  for (int t = 0; t < 2; ++t) {
    const int r = size + t;
    const int gj = t == 0 ? j : j + n;
    T* Lr = L + r * (r + 1) / 2;
    for (int c = 0; c <= r; ++c) {
      const int mc = ((c >> 1) == count) ? j : modes[c >> 1];
      const int gc = (c & 1) ? mc + n : mc;
      T s = Op::from(((gj == gc) ? 1.0 : 0.0) - O[gj * dim + gc]);
      const T* Lc = L + c * (c + 1) / 2;
      for (int u = 0; u < c; ++u) s = Op::fms(s, Lr[u], Lc[u]);
      if (c < r) {
        Lr[c] = Op::div(s, Lc[c]);
      } else {
        if (!Op::pos(s)) return false;
        Lr[r] = Op::sqrt_(s);
      }
    }
  }
  T a = L[size * (size + 1) / 2 + size];
  T b = L[(size + 1) * (size + 2) / 2 + size + 1];
  T ab = Op::mul(a, b);
  detf = Op::mul(ab, ab);
  return true;
}

// One lane's partial torontonian: prefix pattern `pat` over modes [0, g), then all
// 2^(n-g) subsets of modes [g, n).  Returns false (off-domain) on a non-SPD minor.
template <class T>
static __device__ bool tor_lane_subtree(const double* __restrict__ O, int n, int g, uint32_t pat, T* L,
                                 T& total, double& absacc, bool kappa) {
  using Op = TorOps<T>;
  int modes[kTorMaxModes];
  T detat[kTorMaxModes + 1];  // det of the factor with c included modes
  int count = 0;
  detat[0] = Op::from(1.0);
  for (int j = 0; j < g; ++j) {
    if (!((pat >> j) & 1u)) continue;
    modes[count] = j;
    T df;
    if (!tor_append<T>(O, n, j, count, modes, L, df)) return false;
    detat[count + 1] = Op::mul(detat[count], df);
    ++count;
  }
  const int pc = count;
  const int r = n - g;
  total = Op::zero();
  // leaf with all remaining modes excluded
  {
    T c = Op::rsqrt_term(detat[pc]);
    total = ((n - pc) & 1) ? Op::neg(c) : c;
    if (kappa) absacc += fabs(Op::to_d(c));
  }
  const uint64_t nT = 1ull << r;
  for (uint64_t Tm = 1; Tm < nT; ++Tm) {
    // counter bit b <-> mode g + r - 1 - b ; lowest bit = last mode
    const int z = __ffsll((long long)Tm) - 1;
    const int jz = g + r - 1 - z;
    const int above = __popcll((long long)(Tm >> (z + 1)));  // included modes before jz
    const int cnt0 = pc + above;
    modes[cnt0] = jz;
    T df;
    if (!tor_append<T>(O, n, jz, cnt0, modes, L, df)) return false;
    detat[cnt0 + 1] = Op::mul(detat[cnt0], df);
    const int cntl = cnt0 + 1;
    T c = Op::rsqrt_term(detat[cntl]);
    total = ((n - cntl) & 1) ? Op::sub(total, c) : Op::add(total, c);
    if (kappa) absacc += fabs(Op::to_d(c));
  }
  return true;
}

}  // namespace gbsb
