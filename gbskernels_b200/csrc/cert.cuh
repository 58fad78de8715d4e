// cert.cuh -- certified tier: binary64 value + rigorous bound |value - exact| <= bound,
// the bound carried in upward-rounded (directed-rounding) arithmetic per operation.
//
// Model: every binary64 operation o(x, y) returns o(x, y)(1 + d) + a, |d| <= u = 2^-53,
// |a| <= 2^-1074 (subnormal floor, charged as kUfl).  A computed quantity x^ carries a
// radius r with |x^ - x*| <= r, x* the exact-arithmetic value from the exact binary64
// input ("ball arithmetic": the midpoint is the ordinary binary64 computation, the
// radius an upward-rounded running bound).  Reference counterparts:
// core/certified.cu (perm/haf/lhaf recipes), core/tor_recursive.cu:293-431
// (recursive-Cholesky torontonian), core/certified_rounding.cuh (the directed
// rounding helpers; here CUDA's __dadd_ru / __dmul_ru / __ddiv_ru ... are called).
#pragma once

#include "gbs_common.cuh"

namespace gbsb {

// u/(1-u) rounded up: bounds u|x*| by kUc|fl(x)| for a rounded result fl(x) of x*.
constexpr double kUc = 1.1102230246251568e-16;

// Ball in R: midpoint v, radius r.
struct rball {
  double v, r;
};
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
// Certified recursive prefix-Cholesky torontonian, one lane's subtree (same walk as
// tor_lane_subtree in perm_tor.cuh).  L and EL are packed lower-triangular (row r at
// r(r+1)/2); EL[r][c] bounds |L^[r][c] - L*[r][c]|.
//
// Entry (r, c), c <= r, with m = (I - O_S)[r][c] (rounded only on the diagonal):
//   s^ = m - sum_{t<c} L^[r][t] L^[c][t]     (FMA chain, c+1 rounded operations)
//   e_s = e_m + sum_t (EL_rt |L^_ct| + |L^_rt| EL_ct + EL_rt EL_ct)
//         + gamma_{c+1} (|m| + sum_t |L^_rt||L^_ct|) + (c+1) ufl
//   c < r:  L = s^/p^, p^ = L^[c][c] with bound ep < p^:
//           EL = (e_s + |L| ep) / (p^ - ep) + u|L| + ufl
//   c = r:  L = sqrt(s^), certifiable iff s^ - e_s > 0:
//           EL = e_s / sqrt(s^) + u L + ufl   (|sqrt a - sqrt b| = |a-b|/(sqrt a + sqrt b))
//   det factor (l_xx l_pp)^2 and the running det product are real balls; a leaf
//   term 1/sqrt(det) is enclosed by [1/sqrt(D^+e), 1/sqrt(D^-e)] with the bounds
//   computed in outward rounding.  Anything uncertifiable returns false.
__device__ __forceinline__ double gamma_k(int k) { return gamma_ru((double)k, kU); }

__device__ __forceinline__ bool tor_append_cert(const double* __restrict__ O, int n, int j, int count,
                                                const int* modes, double* L, double* EL, rball& detf) {
  const int dim = 2 * n;
  const int size = 2 * count;
  for (int t = 0; t < 2; ++t) {
    const int r = size + t;
    const int gj = t == 0 ? j : j + n;
    double* Lr = L + r * (r + 1) / 2;
    double* ELr = EL + r * (r + 1) / 2;
    for (int c = 0; c <= r; ++c) {
      const int mc = ((c >> 1) == count) ? j : modes[c >> 1];
      const int gc = (c & 1) ? mc + n : mc;
      const double m = ((gj == gc) ? 1.0 : 0.0) - O[gj * dim + gc];
      const double em = (gj == gc) ? ru_add(ru_mul(kU, fabs(m)), kUfl) : 0.0;
      const double* Lc = L + c * (c + 1) / 2;
      const double* ELc = EL + c * (c + 1) / 2;
      double s = m;
      double prop = 0.0, mag = fabs(m);
      for (int u = 0; u < c; ++u) {
        const double lr = Lr[u], lc = Lc[u], er = ELr[u], ec = ELc[u];
        s = fma(-lr, lc, s);
        prop = ru_add(prop, ru_add(ru_mul(er, fabs(lc)), ru_add(ru_mul(fabs(lr), ec), ru_mul(er, ec))));
        mag = ru_fma(fabs(lr), fabs(lc), mag);
      }
      double es = ru_add(ru_add(em, prop), ru_add(ru_mul(gamma_k(c + 1), mag), ru_mul((double)(c + 1), kUfl)));
      if (c < r) {
        const double p = Lc[c], ep = ELc[c];
        if (!(ep < p)) return false;
        const double v = s / p;
        Lr[c] = v;
        const double den = rd_sub(p, ep);
        const double av = ru_mul(fabs(v), 1.0 + 4.0 * kU);  // >= |s^/p^|
        ELr[c] = ru_add(ru_div(ru_add(es, ru_mul(av, ep)), den), ru_add(ru_mul(kU, av), kUfl));
      } else {
        if (!(s > 0.0) || !(rd_sub(s, es) > 0.0)) return false;
        const double v = sqrt(s);
        Lr[r] = v;
        ELr[r] = ru_add(ru_div(es, rd_sqrt(s)), ru_add(ru_mul(kUc, v), kUfl));
      }
    }
  }
  const double a = L[size * (size + 1) / 2 + size], ea = EL[size * (size + 1) / 2 + size];
  const double b = L[(size + 1) * (size + 2) / 2 + size + 1], eb = EL[(size + 1) * (size + 2) / 2 + size + 1];
  // ab = a*b, d = ab*ab, real ball products
  const double ab = a * b;
  double eab = ru_add(ru_add(ru_mul(fabs(a), eb), ru_mul(fabs(b), ea)), ru_mul(ea, eb));
  eab = ru_add(eab, ru_add(ru_mul(kUc, fabs(ab)), kUfl));
  const double d = ab * ab;
  double ed = ru_add(ru_mul(2.0, ru_mul(fabs(ab), eab)), ru_mul(eab, eab));
  ed = ru_add(ed, ru_add(ru_mul(kUc, d), kUfl));
  detf = rball{d, ed};
  return true;
}

__device__ __forceinline__ rball rb_mul(rball x, rball y) {
  rball o;
  o.v = x.v * y.v;
  double r = ru_add(ru_add(ru_mul(fabs(x.v), y.r), ru_mul(fabs(y.v), x.r)), ru_mul(x.r, y.r));
  o.r = ru_add(r, ru_add(ru_mul(kUc, fabs(o.v)), kUfl));
  return o;
}

// Leaf term 1 / sqrt(D), D in [D^ - e, D^ + e], D^ > e.  Returns the computed
// binary64 value and a bound on its distance to 1/sqrt(D*).
__device__ __forceinline__ bool leaf_cert(rball D, rball& term) {
  if (!(D.v > 0.0) || !(rd_sub(D.v, D.r) > 0.0)) return false;
  const double c = 1.0 / sqrt(D.v);
  const double hi = ru_div(1.0, rd_sqrt(rd_sub(D.v, D.r)));
  const double lo = __ddiv_rd(1.0, ru_sqrt(ru_add(D.v, D.r)));
  if (!isfinite(hi) || !isfinite(c)) return false;
  term = rball{c, fmax(ru_add(hi, -c), rd_sub(c, lo) >= 0.0 ? ru_add(c, -lo) : 0.0)};
  return true;
}

static __device__ bool tor_lane_subtree_cert(const double* __restrict__ O, int n, int g, uint32_t pat, double* L,
                                      double* EL, double& total, double& bound) {
  int modes[32];
  rball detat[33];
  int count = 0;
  detat[0] = rball{1.0, 0.0};
  for (int j = 0; j < g; ++j) {
    if (!((pat >> j) & 1u)) continue;
    modes[count] = j;
    rball df;
    if (!tor_append_cert(O, n, j, count, modes, L, EL, df)) return false;
    detat[count + 1] = rb_mul(detat[count], df);
    ++count;
  }
  const int pc = count, r = n - g;
  double tot = 0.0, bnd = 0.0;
  {
    rball t;
    if (!leaf_cert(detat[pc], t)) return false;
    tot = ((n - pc) & 1) ? -t.v : t.v;
    bnd = t.r;
  }
  const uint64_t nT = 1ull << r;
  for (uint64_t Tm = 1; Tm < nT; ++Tm) {
    const int z = __ffsll((long long)Tm) - 1;
    const int jz = g + r - 1 - z;
    const int cnt0 = pc + __popcll((long long)(Tm >> (z + 1)));
    modes[cnt0] = jz;
    rball df;
    if (!tor_append_cert(O, n, jz, cnt0, modes, L, EL, df)) return false;
    detat[cnt0 + 1] = rb_mul(detat[cnt0], df);
    rball t;
    if (!leaf_cert(detat[cnt0 + 1], t)) return false;
    tot = ((n - cnt0 - 1) & 1) ? tot - t.v : tot + t.v;
    bnd = ru_add(ru_add(bnd, t.r), ru_add(ru_mul(kUc, fabs(tot)), kUfl));
  }
  total = tot;
  bound = bnd;
  return true;
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

}  // namespace gbsb
