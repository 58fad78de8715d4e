// cert.cuh -- certified tier: binary64 value + rigorous bound |value - exact| <= bound,
// the bound carried in upward-rounded (directed-rounding) arithmetic per operation.
//
// Model: every binary64 operation o(x, y) returns o(x, y)(1 + d) + a, |d| <= u = 2^-53,
// |a| <= 2^-1074 (subnormal floor, charged as kUfl).  A computed quantity x^ carries a
// radius r with |x^ - x*| <= r, x* the exact-arithmetic value from the exact binary64
// input ("ball arithmetic": the midpoint is the ordinary binary64 computation, the
// radius an upward-rounded running bound).  Reference counterparts:
// core/certified.cu (perm/haf/lhaf recipes), core/certified_rounding.cuh (the
// directed rounding helpers; here CUDA's __dadd_ru / __dmul_ru / __ddiv_ru ... are
// called).  The certified torontonian (reference core/tor_recursive.cu:293-431) uses
// an a-posteriori bound instead and lives in tor_warp.cuh.
#pragma once

#include "gbs_common.cuh"

namespace gbsb {

// u/(1-u) rounded up: bounds u|x*| by kUc|fl(x)| for a rounded result fl(x) of x*.
constexpr double kUc = 1.1102230246251568e-16;

// Ball in C: midpoint z, radius r (bound on the complex modulus of the error).
struct cball {
  cplx z;
  double r;
};

__device__ __forceinline__ double ru_abs_c(cplx z) {
  // upward-rounded |z|: sqrt_ru(re^2 + im^2) with each step rounded up
  return ru_sqrt(ru_fma(z.re, z.re, ru_mul(z.im, z.im)));
}

// x + y: radius rx + ry + u|x^ + y^| (+ underflow floor)
__device__ __forceinline__ cball cb_add(cball x, cball y) {
  cball o;
  o.z = cadd(x.z, y.z);
  o.r = ru_add(ru_add(x.r, y.r), ru_add(ru_mul(kUc, ru_abs_c(o.z)), kUfl));
  return o;
}
__device__ __forceinline__ cball cb_neg(cball x) { return cball{cneg(x.z), x.r}; }
// x * y with the FMA-based complex product: |fl(xy) - xy| <= 4u |x||y| (each
// component a*c - b*d as fma(a, c, -(b*d)) errs by <= 2u(|ac| + |bd|), and
// (|ac|+|bd|)^2 + (|ad|+|bc|)^2 <= 2|x|^2|y|^2).
__device__ __forceinline__ cball cb_mul(cball x, cball y) {
  cball o;
  o.z = cmul(x.z, y.z);
  const double ax = ru_abs_c(x.z), ay = ru_abs_c(y.z);
  double r = ru_add(ru_mul(ax, y.r), ru_mul(ay, x.r));
  r = ru_add(r, ru_mul(x.r, y.r));
  r = ru_add(r, ru_add(ru_mul(4.0 * kU, ru_mul(ax, ay)), 4.0 * kUfl));
  o.r = r;
  return o;
}
__device__ __forceinline__ cball cb_scale(cball x, double s) {  // s exact, |s| >= 1 or a power of 2
  cball o;
  o.z = cscale(x.z, s);
  o.r = ru_add(ru_mul(fabs(s), x.r), ru_add(ru_mul(kUc, ru_abs_c(o.z)), kUfl));
  return o;
}
__device__ __forceinline__ cball cb_div_int(cball x, double j) {  // division by a positive integer
  cball o;
  o.z = cplx{x.z.re / j, x.z.im / j};
  o.r = ru_add(ru_div(x.r, j), ru_add(ru_mul(kUc, ru_abs_c(o.z)), kUfl));
  return o;
}

// Warp butterfly sum of balls (fixed order; every lane gets the result).
__device__ __forceinline__ cball warp_sum_cb(cball b) {
#pragma unroll
  for (int m = 16; m > 0; m >>= 1) {
    cball o{cplx{shfl_xor_d(b.z.re, m), shfl_xor_d(b.z.im, m)}, shfl_xor_d(b.r, m)};
    b = cb_add(b, o);
  }
  return b;
}

// ---------------------------------------------------------------------------------
// Certified Glynn walk of one lane: the binary64 value path of perm_lane_range
// (perm_tor.cuh) operation for operation, each row sum carrying a radius.
//   row-sum update r += (+-2A)[r][col] (exact addend): radius += u|r^new| + ufl
//   row product: balanced tree of ball products (cb_mul), signed ball sum of terms.
template <int NN>
__device__ __forceinline__ cball tree_prod_cb(const cball (&v)[NN]) {
  if constexpr (NN == 1) {
    return v[0];
  } else {
    constexpr int H = NN / 2;
    cball lo[H], hi[NN - H];
#pragma unroll
    for (int i = 0; i < H; ++i) lo[i] = v[i];
#pragma unroll
    for (int i = 0; i < NN - H; ++i) hi[i] = v[H + i];
    return cb_mul(tree_prod_cb<H>(lo), tree_prod_cb<NN - H>(hi));
  }
}

template <int NN>
__device__ __forceinline__ cball perm_lane_range_cert(const double* __restrict__ A2, uint64_t i0, uint64_t R) {
  cball rs[NN];
  const uint64_t g0 = gray_of(i0);
#pragma unroll
  for (int r = 0; r < NN; ++r) {
    cplx s = mkc(0.0, 0.0);
    double rad = 0.0;
#pragma unroll 4
    for (int c = 0; c < NN; ++c) {
      cplx a = ld_c(A2 + (r * NN + c) * 2);
      double sg = (c > 0 && ((g0 >> (c - 1)) & 1ull)) ? -0.5 : 0.5;
      s.re = fma(sg, a.re, s.re);
      s.im = fma(sg, a.im, s.im);
      rad = ru_add(rad, ru_add(ru_mul(kUc, ru_abs_c(s)), kUfl));
    }
    rs[r] = cball{s, rad};
  }
  cball acc;
  {
    cball p = tree_prod_cb<NN>(rs);
    acc = (i0 & 1ull) ? cb_neg(p) : p;
  }
  double sign = (i0 & 1ull) ? -1.0 : 1.0;
  for (uint64_t j = 1; j < R; ++j) {
    const uint64_t i = i0 + j;
    const int k = __ffsll((long long)j) - 1;
    const double step = ((gray_of(i) >> k) & 1ull) ? -1.0 : 1.0;
    const double* col = A2 + (k + 1) * 2;
#pragma unroll
    for (int r = 0; r < NN; ++r) {
      cplx a = ld_c(col + r * NN * 2);
      rs[r].z.re = fma(step, a.re, rs[r].z.re);
      rs[r].z.im = fma(step, a.im, rs[r].z.im);
      rs[r].r = ru_add(rs[r].r, ru_add(ru_mul(kUc, ru_abs_c(rs[r].z)), kUfl));
    }
    sign = -sign;
    cball p = tree_prod_cb<NN>(rs);
    // acc + sign * p, the same rounding as fma(sign, p, acc)
    cball o;
    o.z.re = fma(sign, p.z.re, acc.z.re);
    o.z.im = fma(sign, p.z.im, acc.z.im);
    o.r = ru_add(ru_add(acc.r, p.r), ru_add(ru_mul(kUc, ru_abs_c(o.z)), kUfl));
    acc = o;
  }
  return acc;
}


// ---------------------------------------------------------------------------------
// Certified double-double Glynn walk of one lane: the value path of
// perm_lane_range_dd (perm_tor.cuh) operation for operation, each double-word
// complex carrying a radius that bounds the modulus of its error.  Per-operation
// relative bounds (u = 2^-53; Joldes, Muller and Popescu, "Tight and rigorous error
// bounds for basic building blocks of double-word arithmetic", 2017): the sum of a
// double-word and a double 2u^2, the accurate double-word sum 3u^2/(1-4u), the
// FMA double-word product 5u^2; charged here with slack:
//   every double-word sum (row-sum update, acc +- p, butterfly):
//     radius += 4u^2 (|re| + |im|) of the result
//   complex product of two double-word complexes: per component two products and
//     one sum, <= 9u^2 (|ac| + |bd|) (1 + O(u)); over both components
//     (|a|+|b|)(|c|+|d|) <= 2|x||y|, so 18u^2 |x||y|, charged 21u^2 |x||y|
// plus an absolute underflow term per operation (kUfl, 8 kUfl for a product).
// |z| of a double-word complex is bounded by (|re.hi| + |im.hi|)(1 + 4u).
struct ddball {
  ddc z;
  double r;
};
__device__ __forceinline__ double ddc_mag_up(const ddc& z) {
  return ru_mul(ru_add(fabs(z.re.hi), fabs(z.im.hi)), 1.0 + 4.0 * kU);
}
__device__ __forceinline__ double dd_round_err(const ddc& z) {  // 4u^2 (|re| + |im|)
  return ru_add(ru_mul(4.0 * kU * kU, ddc_mag_up(z)), kUfl);
}
__device__ __forceinline__ ddball ddb_mul(const ddball& x, const ddball& y) {
  ddball o;
  o.z = ddc_mul(x.z, y.z);
  const double mx = ddc_mag_up(x.z), my = ddc_mag_up(y.z);
  double r = ru_add(ru_add(ru_mul(mx, y.r), ru_mul(my, x.r)), ru_mul(x.r, y.r));
  o.r = ru_add(r, ru_add(ru_mul(21.0 * kU * kU, ru_mul(mx, my)), 8.0 * kUfl));
  return o;
}
template <int NN>
__device__ __forceinline__ ddball tree_prod_ddb(const ddball (&v)[NN]) {
  if constexpr (NN == 1) {
    return v[0];
  } else {
    constexpr int H = NN / 2;
    ddball lo[H], hi[NN - H];
#pragma unroll
    for (int i = 0; i < H; ++i) lo[i] = v[i];
#pragma unroll
    for (int i = 0; i < NN - H; ++i) hi[i] = v[H + i];
    return ddb_mul(tree_prod_ddb<H>(lo), tree_prod_ddb<NN - H>(hi));
  }
}

template <int NN>
__device__ __forceinline__ ddball perm_lane_range_certdd(const double* __restrict__ A2, uint64_t i0, uint64_t R) {
  ddball rs[NN];
  const uint64_t g0 = gray_of(i0);
#pragma unroll
  for (int r = 0; r < NN; ++r) {
    ddc s = ddc{dd_make(0.0), dd_make(0.0)};
    double rad = 0.0;
    for (int c = 0; c < NN; ++c) {
      cplx a = ld_c2(A2 + (r * NN + c) * 2);
      double sg = (c > 0 && ((g0 >> (c - 1)) & 1ull)) ? -0.5 : 0.5;  // exact scaling of 2A
      s = ddc{dd_add_d(s.re, sg * a.re), dd_add_d(s.im, sg * a.im)};
      rad = ru_add(rad, dd_round_err(s));
    }
    rs[r] = ddball{s, rad};
  }
  bool neg = (i0 & 1ull) != 0;
  ddball acc;
  {
    ddball p = tree_prod_ddb<NN>(rs);
    acc = ddball{neg ? ddc_neg(p.z) : p.z, p.r};
  }
  for (uint64_t j = 1; j < R; ++j) {
    const uint64_t i = i0 + j;
    const int k = __ffsll((long long)j) - 1;
    const bool minus = ((gray_of(i) >> k) & 1ull) != 0;
    const double* col = A2 + (k + 1) * 2;
#pragma unroll
    for (int r = 0; r < NN; ++r) {
      cplx a = ld_c2(col + r * NN * 2);  // exact 2A
      rs[r].z.re = dd_add_d(rs[r].z.re, minus ? -a.re : a.re);
      rs[r].z.im = dd_add_d(rs[r].z.im, minus ? -a.im : a.im);
      rs[r].r = ru_add(rs[r].r, dd_round_err(rs[r].z));
    }
    neg = !neg;
    ddball p = tree_prod_ddb<NN>(rs);
    acc.z = neg ? ddc_sub(acc.z, p.z) : ddc_add(acc.z, p.z);
    acc.r = ru_add(ru_add(acc.r, p.r), dd_round_err(acc.z));
  }
  return acc;
}

// butterfly of double-word balls (value ops those of warp_sum_ddc)
__device__ __forceinline__ ddball warp_sum_ddb(ddball b) {
#pragma unroll
  for (int m = 16; m > 0; m >>= 1) {
    const ddc o = shfl_xor_ddc(b.z, m);
    const double orr = shfl_xor_d(b.r, m);
    b.z = ddc_add(b.z, o);
    b.r = ru_add(ru_add(b.r, orr), dd_round_err(b.z));
  }
  return b;
}

}  // namespace gbsb
