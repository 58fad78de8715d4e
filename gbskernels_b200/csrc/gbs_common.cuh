// gbs_common.cuh -- shared device primitives for the sm_100a kernels.
//
//   * complex binary64 helpers (the numpy complex128 layout: {re, im})
//   * double-double (DD) arithmetic, written from the published error-free
//     transformations: Knuth's TwoSum (TAOCP vol. 2, 4.2.2), Dekker's Fast2Sum and
//     FMA-based TwoProduct (Dekker 1971; Ogita-Rump-Oishi 2005), and the
//     double-word add / multiply / divide of Hida-Li-Bailey ("QD", 2001) and
//     Joldes-Muller-Popescu (ACM TOMS 2017).
//   * directed-rounding wrappers (CUDA's __dadd_ru / __dmul_ru / __fma_ru ...)
//   * FP64 tensor-core MMA (mma.sync m16n8k4 / m8n8k4 .f64)
//   * status codes shared with the host (include/gbs_b200.h)
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace gbsb {

// ------------------------------------------------------------------ status
// Per-instance status words written by the kernels (0 = ok). The host maps them
// to the reference's value conventions (NaN for off-domain / uncertifiable).
enum : int {
  kStOk = 0,
  kStOffDomain = 1,     // torontonian leading minor not positive definite
  kStUncertified = 2,   // certified bound could not be established
  kStTooLarge = 3,      // size above the compiled cap
  kStTimeout = 4,       // bounded spin gave up (queue kernels)
};

// ------------------------------------------------------------------ complex
struct cplx {
  double re, im;
};
__host__ __device__ __forceinline__ cplx mkc(double r, double i) { return cplx{r, i}; }
__host__ __device__ __forceinline__ cplx cadd(cplx a, cplx b) { return cplx{a.re + b.re, a.im + b.im}; }
__host__ __device__ __forceinline__ cplx csub(cplx a, cplx b) { return cplx{a.re - b.re, a.im - b.im}; }
__host__ __device__ __forceinline__ cplx cmul(cplx a, cplx b) {
  return cplx{fma(a.re, b.re, -a.im * b.im), fma(a.re, b.im, a.im * b.re)};
}
// acc + a*b with fused operations
__host__ __device__ __forceinline__ cplx cfma(cplx a, cplx b, cplx acc) {
  acc.re = fma(a.re, b.re, acc.re);
  acc.re = fma(-a.im, b.im, acc.re);
  acc.im = fma(a.re, b.im, acc.im);
  acc.im = fma(a.im, b.re, acc.im);
  return acc;
}
__host__ __device__ __forceinline__ cplx cscale(cplx a, double s) { return cplx{a.re * s, a.im * s}; }
__host__ __device__ __forceinline__ cplx cneg(cplx a) { return cplx{-a.re, -a.im}; }
__device__ __forceinline__ double cabs_fast(cplx a) { return sqrt(fma(a.re, a.re, a.im * a.im)); }

// ------------------------------------------------------------------ double-double
struct dd {
  double hi, lo;
};
struct ddc {
  dd re, im;
};

// TwoSum (Knuth): s + e == a + b exactly, no ordering assumption.
__host__ __device__ __forceinline__ double two_sum(double a, double b, double& e) {
  double s = a + b;
  double bv = s - a;
  double av = s - bv;
  e = (a - av) + (b - bv);
  return s;
}
// Fast2Sum (Dekker): valid when |a| >= |b| (or a == 0).
__host__ __device__ __forceinline__ double fast_two_sum(double a, double b, double& e) {
  double s = a + b;
  e = b - (s - a);
  return s;
}
// TwoProduct with a fused multiply-add: p + e == a * b exactly.
__host__ __device__ __forceinline__ double two_prod(double a, double b, double& e) {
  double p = a * b;
  e = fma(a, b, -p);
  return p;
}

__host__ __device__ __forceinline__ dd dd_make(double a) { return dd{a, 0.0}; }
__host__ __device__ __forceinline__ dd dd_neg(dd a) { return dd{-a.hi, -a.lo}; }

// Accurate double-word sum (two TwoSums; relative error ~3u^2 even under
// cancellation, the variant recommended for alternating sums).
__host__ __device__ __forceinline__ dd dd_add(dd a, dd b) {
  double e1, e2;
  double s = two_sum(a.hi, b.hi, e1);
  double t = two_sum(a.lo, b.lo, e2);
  e1 += t;
  s = fast_two_sum(s, e1, e1);
  e1 += e2;
  s = fast_two_sum(s, e1, e1);
  return dd{s, e1};
}
__host__ __device__ __forceinline__ dd dd_sub(dd a, dd b) { return dd_add(a, dd_neg(b)); }
__host__ __device__ __forceinline__ dd dd_add_d(dd a, double b) {
  double e;
  double s = two_sum(a.hi, b, e);
  e += a.lo;
  s = fast_two_sum(s, e, e);
  return dd{s, e};
}
// Double-word product (FMA based).
__host__ __device__ __forceinline__ dd dd_mul(dd a, dd b) {
  double e;
  double p = two_prod(a.hi, b.hi, e);
  e = fma(a.hi, b.lo, e);
  e = fma(a.lo, b.hi, e);
  p = fast_two_sum(p, e, e);
  return dd{p, e};
}
__host__ __device__ __forceinline__ dd dd_mul_d(dd a, double b) {
  double e;
  double p = two_prod(a.hi, b, e);
  e = fma(a.lo, b, e);
  p = fast_two_sum(p, e, e);
  return dd{p, e};
}
// Division by a double: quotient digit, exact remainder via TwoProduct, correction.
__host__ __device__ __forceinline__ dd dd_div_d(dd a, double b) {
  double q1 = a.hi / b;
  double pe;
  double p = two_prod(q1, b, pe);
  dd r = dd_sub(a, dd{p, pe});
  double q2 = r.hi / b;
  double e;
  double q = fast_two_sum(q1, q2, e);
  return dd{q, e};
}
// Division a / b (three quotient digits, renormalised).
__host__ __device__ __forceinline__ dd dd_div(dd a, dd b) {
  double q1 = a.hi / b.hi;
  dd r = dd_sub(a, dd_mul_d(b, q1));
  double q2 = r.hi / b.hi;
  r = dd_sub(r, dd_mul_d(b, q2));
  double q3 = r.hi / b.hi;
  double e;
  double q = fast_two_sum(q1, q2, e);
  return dd_add(dd{q, e}, dd{q3, 0.0});
}
// Square root: binary64 seed y0 = sqrt(a.hi), one Newton correction
// y = y0 + (a - y0^2) / (2 y0) carried in double-word.
__host__ __device__ __forceinline__ dd dd_sqrt(dd a) {
  if (!(a.hi > 0.0)) return dd{0.0, 0.0};
  double y0 = sqrt(a.hi);
  double e;
  double sq = two_prod(y0, y0, e);
  dd r = dd_sub(a, dd{sq, e});
  double corr = r.hi / (2.0 * y0);
  double lo;
  double hi = fast_two_sum(y0, corr, lo);
  return dd{hi, lo};
}

__host__ __device__ __forceinline__ ddc ddc_make(cplx a) { return ddc{dd_make(a.re), dd_make(a.im)}; }
__host__ __device__ __forceinline__ ddc ddc_add(ddc a, ddc b) { return ddc{dd_add(a.re, b.re), dd_add(a.im, b.im)}; }
__host__ __device__ __forceinline__ ddc ddc_sub(ddc a, ddc b) { return ddc{dd_sub(a.re, b.re), dd_sub(a.im, b.im)}; }
__host__ __device__ __forceinline__ ddc ddc_neg(ddc a) { return ddc{dd_neg(a.re), dd_neg(a.im)}; }
__host__ __device__ __forceinline__ ddc ddc_mul(ddc a, ddc b) {
  return ddc{dd_sub(dd_mul(a.re, b.re), dd_mul(a.im, b.im)),
             dd_add(dd_mul(a.re, b.im), dd_mul(a.im, b.re))};
}
__host__ __device__ __forceinline__ ddc ddc_mul_d(ddc a, double s) { return ddc{dd_mul_d(a.re, s), dd_mul_d(a.im, s)}; }
__host__ __device__ __forceinline__ ddc ddc_div_d(ddc a, double s) { return ddc{dd_div_d(a.re, s), dd_div_d(a.im, s)}; }
// Collapse to binary64 (round-to-nearest of hi + lo).
__host__ __device__ __forceinline__ cplx ddc_to_c(ddc a) { return cplx{a.re.hi + a.re.lo, a.im.hi + a.im.lo}; }

// ------------------------------------------------------------------ directed rounding
// Upward / downward rounded operations for the certified bound accumulators.
__device__ __forceinline__ double ru_add(double a, double b) { return __dadd_ru(a, b); }
__device__ __forceinline__ double ru_mul(double a, double b) { return __dmul_ru(a, b); }
__device__ __forceinline__ double ru_fma(double a, double b, double c) { return __fma_ru(a, b, c); }
__device__ __forceinline__ double ru_div(double a, double b) { return __ddiv_ru(a, b); }
__device__ __forceinline__ double rd_add(double a, double b) { return __dadd_rd(a, b); }
__device__ __forceinline__ double rd_sub(double a, double b) { return __dsub_rd(a, b); }
__device__ __forceinline__ double rd_mul(double a, double b) { return __dmul_rd(a, b); }
__device__ __forceinline__ double rd_sqrt(double a) { return __dsqrt_rd(a); }
__device__ __forceinline__ double ru_sqrt(double a) { return __dsqrt_ru(a); }

// Unit roundoff of binary64 and a conservative absolute underflow term per operation.
constexpr double kU = 1.1102230246251565e-16;       // 2^-53
constexpr double kUfl = 8e-323;                      // 16 * 2^-1074
// gamma_k = k u / (1 - k u), rounded upward.
__device__ __forceinline__ double gamma_ru(double k, double u) {
  double ku = ru_mul(k, u);
  return ru_div(ku, rd_sub(1.0, ku));
}

// ------------------------------------------------------------------ warp helpers
__device__ __forceinline__ double shfl_xor_d(double v, int m) { return __shfl_xor_sync(0xffffffffu, v, m); }
__device__ __forceinline__ double warp_sum_d(double v) {
#pragma unroll
  for (int m = 16; m > 0; m >>= 1) v += shfl_xor_d(v, m);
  return v;
}
// Upward-rounded warp sum (every lane gets the same value).
__device__ __forceinline__ double warp_sum_ru(double v) {
#pragma unroll
  for (int m = 16; m > 0; m >>= 1) v = ru_add(v, shfl_xor_d(v, m));
  return v;
}
__device__ __forceinline__ double warp_max_d(double v) {
#pragma unroll
  for (int m = 16; m > 0; m >>= 1) v = fmax(v, shfl_xor_d(v, m));
  return v;
}

// ------------------------------------------------------------------ FP64 tensor core MMA
// D(16x8) = A(16x4, row) * B(4x8, col) + C, binary64 operands.  Fragment layout
// (PTX ISA, mma .m16n8k4 .f64):  g = lane/4, t = lane%4;
//   a0 = A[g][t], a1 = A[g+8][t];  b0 = B[t][g];
//   c0 = C[g][2t], c1 = C[g][2t+1], c2 = C[g+8][2t], c3 = C[g+8][2t+1].
// The mma helpers are plain (non-volatile) asm: they have no side effects beyond
// their outputs, so the compiler may schedule them like arithmetic.
__device__ __forceinline__ void dmma_m16n8k4(double (&d)[4], double a0, double a1, double b0) {
  asm(
      "mma.sync.aligned.m16n8k4.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, {%4,%5}, {%6}, {%0,%1,%2,%3};\n"
      : "+d"(d[0]), "+d"(d[1]), "+d"(d[2]), "+d"(d[3])
      : "d"(a0), "d"(a1), "d"(b0));
}

// D += A B with m16n8k8 (A: rows g / g+8, columns t4 / t4+4; B: rows t4 / t4+4,
// column g): the work of two consecutive m16n8k4 steps in one instruction.
__device__ __forceinline__ void dmma_m16n8k8(double (&d)[4], double a0, double a1, double a2, double a3, double b0,
                                             double b1) {
  asm(
      "mma.sync.aligned.m16n8k8.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, {%0,%1,%2,%3};\n"
      : "+d"(d[0]), "+d"(d[1]), "+d"(d[2]), "+d"(d[3])
      : "d"(a0), "d"(a1), "d"(a2), "d"(a3), "d"(b0), "d"(b1));
}

// 16-byte complex loads / stores (shared or global memory, 16-byte aligned).
__device__ __forceinline__ cplx ld_c(const double* p) {
  double2 v = *reinterpret_cast<const double2*>(p);
  return cplx{v.x, v.y};
}
__device__ __forceinline__ cplx ld_c2(const double* p) { return ld_c(p); }
__device__ __forceinline__ void st_c(double* p, cplx v) {
  *reinterpret_cast<double2*>(p) = make_double2(v.re, v.im);
}
__device__ __forceinline__ cplx warp_sum_c(cplx v) { return cplx{warp_sum_d(v.re), warp_sum_d(v.im)}; }
__device__ __forceinline__ ddc ld_ddc(const double* p) {
  double4 v = *reinterpret_cast<const double4*>(p);
  return ddc{dd{v.x, v.y}, dd{v.z, v.w}};
}
__device__ __forceinline__ void st_ddc(double* p, ddc v) {
  *reinterpret_cast<double4*>(p) = make_double4(v.re.hi, v.re.lo, v.im.hi, v.im.lo);
}
// DD shuffle-xor and warp sum (fixed butterfly order).
__device__ __forceinline__ ddc shfl_xor_ddc(ddc v, int m) {
  return ddc{dd{shfl_xor_d(v.re.hi, m), shfl_xor_d(v.re.lo, m)}, dd{shfl_xor_d(v.im.hi, m), shfl_xor_d(v.im.lo, m)}};
}
__device__ __forceinline__ ddc warp_sum_ddc(ddc v) {
#pragma unroll
  for (int m = 16; m > 0; m >>= 1) v = ddc_add(v, shfl_xor_ddc(v, m));
  return v;
}

// Combinatorics ---------------------------------------------------------------
__host__ __device__ __forceinline__ uint64_t gray_of(uint64_t i) { return i ^ (i >> 1); }

}  // namespace gbsb
