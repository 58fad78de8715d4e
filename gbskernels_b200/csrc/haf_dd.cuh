// haf_dd.cuh -- hafnian / loop hafnian power trace in complex double-double (the
// "dd" precision tier), one warp per subset, SIMT.
//
// Same algorithm and the same trace identities as haf_pt.cuh (reference:
// core/hafnian_dd.cu:34-107, core/loop_hafnian_dd.cu:40-113, cpu_ref/hafnian.py:101-129),
// with every add / multiply in double-double.  There is no double-double tensor
// instruction, so the strip product runs on the FP64 pipe: lane (row i = lane & 15,
// column half = lane >> 4) forms row i of strip(C^{a+1}) for its half of the columns.
//
// Certified double-double tier (CERT; reference counterpart
// core/certified_dd.cu:216-328, which stops at N = 16): the value is this walk
// operation for operation (bit-identical to the dd tier); the radius is an a-priori
// bound of the same form as the binary64 certificate (haf_pt.cuh), with the
// double-word per-operation bounds: a complex double-word product errs by at most
// 21u^2 |x||y| and a sum by 4u^2 (|re| + |im|) <= 6u^2 |z| of its result (u = 2^-53),
// so a sequential sum of L products of computed operands errs by at most
// zeta_L = (1 + 6u^2)^L (1 + 21u^2) - 1 times the sum of |products|.  With
// M_a = |C|^a (computed on the tensor cores by the binary64 bound path and inflated
// by phi_a), E_a = |P^_a - C^a| <= c_a M_a, c_{a+1} = c_a + zeta_s (1 + c_a); trace
// and loop-term errors follow from the upward-rounded sums sum M_a M_b; the Newton
// recurrence runs in double-word balls, each division certified a posteriori from
// its residual.
#pragma once

#include "gbs_common.cuh"
#include "haf_pt.cuh"

namespace gbsb {

struct HafDDLayout {
  int smax;
  int c_off, p0_off, p1_off, y_off, d_off, gi_off, acc_off, total;  // doubles
  // certified tier only: |C| and the bound-path power (binary64, the strides of
  // haf_pt.cuh), row bounds, trace / loop bound sums, d in binary64
  int ca_off, m_off, ym_off, bt_off, dv_off;
};
// Row stride (doubles) of the double-word power buffers for a subset of side s: at
// least the row's 4 s doubles and == 4 (mod 16), so consecutive rows start 32 bytes
// apart modulo 128 and every complex double word stays 32-byte aligned (ld_ddc is
// one 32-byte load).  The strip product reads one complex double word of each of
// the 16 rows at a time: with rows a multiple of 128 bytes long (s a multiple of 4)
// all 16 fell on the same banks, 16 wavefronts per load; 32 bytes apart they fill
// each 128-byte wavefront four at a time, the minimum of 4.
__host__ __device__ inline int haf_dd_prow(int s) { return 4 * s + ((4 - 4 * s) & 15); }
__host__ __device__ inline int haf_dd_prow_max(int smax) {
  int m = 0;
  for (int s = 2; s <= smax; s += 2) m = m > haf_dd_prow(s) ? m : haf_dd_prow(s);
  return m;
}

__host__ __device__ inline HafDDLayout haf_dd_layout(int smax, bool cert = false) {
  HafDDLayout L;
  if (smax < 2) smax = 2;
  L.smax = smax;
  int h = (smax / 2 + 1) / 2;
  L.c_off = 0;
  L.p0_off = L.c_off + smax * smax * 4;
  L.p1_off = L.p0_off + 16 * haf_dd_prow_max(smax);
  L.y_off = L.p1_off + 16 * haf_dd_prow_max(smax);
  L.d_off = L.y_off + 16 * (h + 1) * 4;
  L.gi_off = L.d_off + 32 * 4;
  L.acc_off = L.gi_off + 16;
  L.total = L.acc_off + 4 * (kHafMaxPairs + 1) * 4;
  L.total = (L.total + 3) & ~3;  // 32-byte multiple
  L.ca_off = L.m_off = L.ym_off = L.bt_off = L.dv_off = 0;
  if (cert) {
    const int rows = 16 * haf_strips(smax), cs = haf_c_stride(smax), ps = haf_p_stride(smax, smax > 16);
    L.ca_off = L.total;
    L.m_off = L.ca_off + rows * cs * 2;
    L.ym_off = L.m_off + rows * ps * 2;
    L.bt_off = L.ym_off + rows * (h + 1);
    L.dv_off = L.bt_off + 2 * (kHafMaxPairs + 2);
    L.total = L.dv_off + 32 * 2;
    L.total = (L.total + 3) & ~3;
  }
  return L;
}

// zeta_L = (1 + 6u^2)^L (1 + em) - 1, upward: x = L 6u^2 + em <= 1e-28, and
// x e^x <= x (1 + 2^-52).
__device__ __forceinline__ double dd_zeta(double L, double em) {
  return ru_mul(ru_add(ru_mul(L, 6.0 * kU * kU), em), 1.0000000000000002);
}
__device__ __forceinline__ ddball ddb_add(const ddball& x, const ddball& y) {
  ddball o;
  o.z = ddc_add(x.z, y.z);
  o.r = ru_add(ru_add(x.r, y.r), dd_round_err(o.z));
  return o;
}
// x / j for a small positive integer j: the value of ddc_div_d; the error of the
// quotient from the residual r = x - q j (|x - q j| <= |r^| + 4u^2 (j|q| + |r^|)).
__device__ __forceinline__ ddball ddb_div_int(const ddball& x, double j) {
  ddball o;
  o.z = ddc_div_d(x.z, j);
  const ddc qj = ddc_mul_d(o.z, j);
  const ddc r = ddc_sub(x.z, qj);
  const double mr = ddc_mag_up(r);
  double e = ru_add(mr, ru_mul(4.0 * kU * kU, ru_add(ddc_mag_up(qj), mr)));
  e = ru_add(e, 4.0 * kUfl);
  o.r = ru_div(ru_add(x.r, e), j);
  return o;
}

__device__ __forceinline__ ddc ddc_zero() { return ddc{dd_make(0.0), dd_make(0.0)}; }

__device__ __forceinline__ ddc strip_pair_trace_dd(const double* X, const double* Y, int rows, int s,
                                                   int lane) {
  ddc acc = ddc_zero();
  const int tot = rows * s, prow = haf_dd_prow(s);
  for (int e = lane; e < tot; e += 32) {
    int i = e / s, t = e - i * s;
    acc = ddc_add(acc, ddc_mul(ld_ddc(X + i * prow + t * 4), ld_ddc(Y + (i ^ 1) * prow + (t ^ 1) * 4)));
  }
  return warp_sum_ddc(acc);
}

__device__ __forceinline__ void strip_matvec_dd(const double* P, const double* Dv, double* Y, int col,
                                                int hp1, int rows, int s, int lane) {
  const int i = lane >> 1, half = lane & 1;
  const int prow = haf_dd_prow(s);
  ddc acc = ddc_zero();
  if (i < rows)
    for (int t = half; t < s; t += 2) acc = ddc_add(acc, ddc_mul(ld_ddc(P + i * prow + t * 4), ld_ddc(Dv + t * 4)));
  acc = ddc_add(acc, shfl_xor_ddc(acc, 1));
  if (half == 0 && i < 16) st_ddc(Y + (i * hp1 + col) * 4, i < rows ? acc : ddc_zero());
}

template <bool CERT>
static __device__ ddball haf_subset_term_dd(const double* __restrict__ A, int N, int n, uint32_t mask, bool loop,
                                            double* ws, const HafDDLayout& Lw, int lane) {
  const int m = __popc(mask);
  if (m == 0) return ddball{ddc{dd_make(n == 0 ? 1.0 : 0.0), dd_make(0.0)}, 0.0};
  const int s = 2 * m;
  const int h = (n + 1) / 2, hp1 = h + 1;
  double* Cs = ws + Lw.c_off;
  double* P0 = ws + Lw.p0_off;
  double* P1 = ws + Lw.p1_off;
  double* Y = ws + Lw.y_off;
  double* Dv = ws + Lw.d_off;
  int* gi = reinterpret_cast<int*>(ws + Lw.gi_off);
  double* acc_p = ws + Lw.acc_off;
  double* acc_v = acc_p + (kHafMaxPairs + 1) * 4;
  double* kg = acc_v + (kHafMaxPairs + 1) * 4;
  double* ev = kg + (kHafMaxPairs + 1) * 4;

  if (lane < s) {
    uint32_t mm = mask;
    for (int u = 0; u < (lane >> 1); ++u) mm &= mm - 1;
    gi[lane] = 2 * (__ffs(mm) - 1) + (lane & 1);
  }
  __syncwarp();
  bool tiny_halving = false;  // certified: a halving that may have rounded (see below)
  for (int e = lane; e < s * s; e += 32) {
    int r = e / s, c = e - r * s;
    int rr = gi[r], cc = gi[c ^ 1];
    ddc v = ddc_zero();
    if (loop || rr != cc) {
      // the symmetric part (A + A^T)/2 exactly, as a double word: TwoSum of the two
      // entries, halved (the half-power identities need B_S symmetric)
      const cplx x = ld_c(A + ((size_t)rr * N + cc) * 2), y = ld_c(A + ((size_t)cc * N + rr) * 2);
      double er, ei;
      const double sr = two_sum(x.re, y.re, er), si = two_sum(x.im, y.im, ei);
      v = ddc{dd{0.5 * sr, 0.5 * er}, dd{0.5 * si, 0.5 * ei}};
      if (CERT && (2.0 * v.re.lo != er || 2.0 * v.im.lo != ei || 2.0 * v.re.hi != sr || 2.0 * v.im.hi != si))
        tiny_halving = true;
    }
    st_ddc(Cs + e * 4, v);
  }
  if (loop && lane < s) st_ddc(Dv + lane * 4, ddc_make(ld_c(A + ((size_t)gi[lane] * N + gi[lane]) * 2)));
  for (int k = lane; k <= n; k += 32) {
    st_ddc(acc_p + 4 * k, ddc_zero());
    st_ddc(acc_v + 4 * k, ddc_zero());
  }
  // certified: |C| and d in binary64 for the bound path (strides of haf_pt.cuh)
  const int cs = haf_c_stride(s), ps = haf_p_stride(s, Lw.smax > 16), brows = 16 * haf_strips(s);
  double* Ca = ws + Lw.ca_off;
  double* M = ws + Lw.m_off;
  double* Ym = ws + Lw.ym_off;
  double* bT = ws + Lw.bt_off;            // trace bound sums T[k]
  double* bV = bT + (kHafMaxPairs + 2);   // loop bound sums V[k]
  double* Dv64 = ws + Lw.dv_off;
  if constexpr (CERT) {
    const int ccols = (((2 * s + 7) >> 3) << 2);
    for (int e = lane; e < brows * ccols; e += 32) {
      const int r = e / ccols, c = e - r * ccols;
      double a = 0.0;
      if (r < s && c < s) {
        const int rr = gi[r], cc = gi[c ^ 1];
        // >= |(A_rc + A_cr) / 2|, the modulus of the staged double-word entry
        if (loop || rr != cc)
          a = ru_mul(0.5, ru_add(ru_abs_c(ld_c(A + ((size_t)rr * N + cc) * 2)),
                                 ru_abs_c(ld_c(A + ((size_t)cc * N + rr) * 2))));
      }
      st_c(Ca + (r * cs + c) * 2, mkc(a, 0.0));
    }
    st_c(Dv64 + lane * 2, (loop && lane < s) ? ld_c(A + ((size_t)gi[lane] * N + gi[lane]) * 2) : mkc(0.0, 0.0));
    for (int k = lane; k <= n + 1; k += 32) { bT[k] = 0.0; bV[k] = 0.0; }
  }
  __syncwarp();
  {
    ddc t = lane < s ? ld_ddc(Cs + (lane * s + lane) * 4) : ddc_zero();
    t = warp_sum_ddc(t);
    if (lane == 0) st_ddc(acc_p + 4, t);
  }
  if constexpr (CERT) {
    double a1 = lane < s ? ld_c(Ca + (lane * cs + lane) * 2).re : 0.0;
    a1 = warp_sum_ru(a1);
    if (lane == 0) bT[1] = a1;
    if (loop && lane < brows) Ym[lane * hp1] = lane < s ? ru_abs_c(ld_c(Dv64 + lane * 2)) : 0.0;
  }
  const int nstrips = (s + 15) >> 4;
  for (int st = 0; st < nstrips; ++st) {
    const int r0 = st * 16;
    const int rows = min(16, s - r0);
    double* Pa = P0;
    double* Pb = P1;
    const int prow = haf_dd_prow(s);
    for (int e = lane; e < 16 * s; e += 32) {
      int i = e / s;
      st_ddc(Pa + i * prow + (e - i * s) * 4, i < rows ? ld_ddc(Cs + ((r0 + i) * s + (e - i * s)) * 4) : ddc_zero());
    }
    __syncwarp();
    {
      ddc t = strip_pair_trace_dd(Pa, Pa, rows, s, lane);
      if (lane == 0 && 2 <= n) st_ddc(acc_p + 8, ddc_add(ld_ddc(acc_p + 8), t));
    }
    if (loop) {
      if (lane < 16) st_ddc(Y + (lane * hp1) * 4, lane < rows ? ld_ddc(Dv + (r0 + lane) * 4) : ddc_zero());
      strip_matvec_dd(Pa, Dv, Y, 1, hp1, rows, s, lane);
    }
    __syncwarp();
    for (int a = 2; a <= h; ++a) {
      // Pb = Pa * C  (SIMT double-double)
      {
        const int i = lane & 15, half = lane >> 4;
        const int j0 = half * (s >> 1), j1 = j0 + (s >> 1);
        if (i < rows) {
          for (int j = j0; j < j1; ++j) {
            ddc acc = ddc_zero();
            for (int t = 0; t < s; ++t) acc = ddc_add(acc, ddc_mul(ld_ddc(Pa + i * prow + t * 4), ld_ddc(Cs + (t * s + j) * 4)));
            st_ddc(Pb + i * prow + j * 4, acc);
          }
        }
      }
      __syncwarp();
      ddc todd = strip_pair_trace_dd(Pb, Pa, rows, s, lane);
      ddc tev = strip_pair_trace_dd(Pb, Pb, rows, s, lane);
      if (lane == 0) {
        if (2 * a - 1 <= n) st_ddc(acc_p + 4 * (2 * a - 1), ddc_add(ld_ddc(acc_p + 4 * (2 * a - 1)), todd));
        if (2 * a <= n) st_ddc(acc_p + 4 * (2 * a), ddc_add(ld_ddc(acc_p + 4 * (2 * a)), tev));
      }
      if (loop) strip_matvec_dd(Pb, Dv, Y, a, hp1, rows, s, lane);
      __syncwarp();
      double* tmp = Pa; Pa = Pb; Pb = tmp;
    }
    if (loop) {
      for (int k = 1; k <= n; ++k) {
        const int aa = (k - 1) >> 1, bb = k - 1 - aa;
        ddc t = ddc_zero();
        if (lane < rows) t = ddc_mul(ld_ddc(Y + ((lane ^ 1) * hp1 + aa) * 4), ld_ddc(Y + (lane * hp1 + bb) * 4));
        t = warp_sum_ddc(t);
        if (lane == 0) st_ddc(acc_v + 4 * k, ddc_add(ld_ddc(acc_v + 4 * k), ddc_mul_d(t, 0.5)));
      }
    }
    __syncwarp();
  }
  double rad = 0.0;
  if constexpr (CERT) {
    // bound path: powers of |C| on the tensor cores (binary64, upward-rounded sums)
    if (s <= 16) haf_bound_powers<4, 1>(Ca, M, Ym, Dv64, bT, s, cs, ps, n, h, loop, lane);
    else haf_bound_powers<8, 2>(Ca, M, Ym, Dv64, bT, s, cs, ps, n, h, loop, lane);
    __syncwarp();
    if (loop) {
      for (int k = 1; k <= n; ++k) {
        const int aa = (k - 1) >> 1, bb = k - 1 - aa;
        double vb = lane < s ? ru_mul(Ym[(lane ^ 1) * hp1 + aa], Ym[lane * hp1 + bb]) : 0.0;
        vb = warp_sum_ru(vb);
        if (lane == 0) bV[k] = vb;
      }
    }
    __syncwarp();
    if (lane == 0) {
      const double em = 21.0 * kU * kU;
      const double zp = dd_zeta((double)s, em);             // one element of P^_a C
      const double zt = dd_zeta(32.0 * 16 / 32 + 5 + 2, em);  // trace: <= 16 per lane, butterfly, strips
      const double zy = dd_zeta((double)(s / 2 + 1), em);   // y_a = P^_a d: half a row + the partner
      const double zv = dd_zeta(1.0 + 5 + 2, em);           // v_k: butterfly over rows, strips
      const double g2s = gamma_ru((double)(2 * s), 2.0 * kU);  // the binary64 bound path (|C| powers)
      double ca[kHafMaxPow + 2], ph[kHafMaxPow + 2], ka[kHafMaxPow + 2];
      ca[0] = 0.0; ph[0] = 1.0; ca[1] = 0.0; ph[1] = 1.0;
      for (int a = 1; a <= h; ++a) {
        ca[a + 1] = ru_add(ca[a], ru_mul(zp, ru_add(1.0, ca[a])));
        ph[a + 1] = ru_div(ph[a], rd_sub(1.0, g2s));
      }
      ka[0] = 0.0;
      for (int a = 1; a <= h; ++a) ka[a] = ru_add(ca[a], ru_mul(zy, ru_add(1.0, ca[a])));
      ddball kgb[kHafMaxPairs + 1];
      for (int k = 1; k <= n; ++k) {
        double ep;
        if (k == 1) {
          ep = ru_mul(dd_zeta(5.0, 0.0), bT[1]);
        } else if ((k & 1) == 0) {
          const int a = k / 2;
          const double f = ru_add(ru_add(ru_mul(2.0, ca[a]), ru_mul(ca[a], ca[a])),
                                  ru_mul(zt, ru_mul(ru_add(1.0, ca[a]), ru_add(1.0, ca[a]))));
          ep = ru_mul(ru_mul(f, ru_mul(ph[a], ph[a])), bT[k]);
        } else {
          const int a = (k + 1) / 2;
          const double f = ru_add(ru_add(ru_add(ca[a], ca[a - 1]), ru_mul(ca[a], ca[a - 1])),
                                  ru_mul(zt, ru_mul(ru_add(1.0, ca[a]), ru_add(1.0, ca[a - 1]))));
          ep = ru_mul(ru_mul(f, ru_mul(ph[a], ph[a - 1])), bT[k]);
        }
        // kg_k = p_k / 2 (exact scaling) + k v_k
        ddball g{ddc_mul_d(ld_ddc(acc_p + 4 * k), 0.5), ru_add(ru_mul(0.5, ep), kUfl)};
        if (loop) {
          const int aa = (k - 1) >> 1, bb = k - 1 - aa;
          const double f = ru_add(ru_add(ru_add(ka[aa], ka[bb]), ru_mul(ka[aa], ka[bb])),
                                  ru_mul(zv, ru_mul(ru_add(1.0, ka[aa]), ru_add(1.0, ka[bb]))));
          const double evb = ru_mul(0.5, ru_mul(ru_mul(f, ru_mul(ph[aa], ph[bb])), bV[k]));
          const ddc kv = ddc_mul_d(ld_ddc(acc_v + 4 * k), (double)k);
          const ddball vb{kv, ru_add(ru_mul((double)k, evb), dd_round_err(kv))};
          g = ddb_add(g, vb);
        }
        kgb[k] = g;
        st_ddc(kg + 4 * k, g.z);
      }
      ddball e[kHafMaxPairs + 1];
      e[0] = ddball{ddc{dd_make(1.0), dd_make(0.0)}, 0.0};
      for (int j = 1; j <= n; ++j) {
        ddball acc{ddc_zero(), 0.0};
        for (int k = 1; k <= j; ++k) acc = ddb_add(acc, ddb_mul(kgb[k], e[j - k]));
        e[j] = ddb_div_int(acc, (double)j);
      }
      st_ddc(ev + 4 * n, e[n].z);
      bT[0] = e[n].r;
    }
    __syncwarp();
    rad = __any_sync(0xffffffffu, tiny_halving) ? INFINITY : bT[0];
  } else {
    if (lane == 0) {
      for (int k = 1; k <= n; ++k) {
        ddc g = ddc_mul_d(ld_ddc(acc_p + 4 * k), 0.5);
        if (loop) g = ddc_add(g, ddc_mul_d(ld_ddc(acc_v + 4 * k), (double)k));
        st_ddc(kg + 4 * k, g);
      }
      st_ddc(ev, ddc{dd_make(1.0), dd_make(0.0)});
      for (int j = 1; j <= n; ++j) {
        ddc acc = ddc_zero();
        for (int k = 1; k <= j; ++k) acc = ddc_add(acc, ddc_mul(ld_ddc(kg + 4 * k), ld_ddc(ev + 4 * (j - k))));
        st_ddc(ev + 4 * j, ddc_div_d(acc, (double)j));
      }
    }
  }
  __syncwarp();
  ddc coeff = ld_ddc(ev + 4 * n);
  __syncwarp();
  return ddball{((n - m) & 1) ? ddc_neg(coeff) : coeff, rad};
}

}  // namespace gbsb
