// haf_dd.cuh -- hafnian / loop hafnian power trace in complex double-double (the
// "dd" precision tier), one warp per subset, SIMT.
//
// Same algorithm and the same trace identities as haf_pt.cuh (reference:
// core/hafnian_dd.cu:34-107, core/loop_hafnian_dd.cu:40-113, cpu_ref/hafnian.py:101-129),
// with every add / multiply in double-double.  There is no double-double tensor
// instruction, so the strip product runs on the FP64 pipe: lane (row i = lane & 15,
// column half = lane >> 4) forms row i of strip(C^{a+1}) for its half of the columns.
#pragma once

#include "gbs_common.cuh"
#include "haf_pt.cuh"

namespace gbsb {

struct HafDDLayout {
  int smax;
  int c_off, p0_off, p1_off, y_off, d_off, gi_off, acc_off, total;  // doubles
};
__host__ __device__ inline HafDDLayout haf_dd_layout(int smax) {
  HafDDLayout L;
  if (smax < 2) smax = 2;
  L.smax = smax;
  int h = (smax / 2 + 1) / 2;
  L.c_off = 0;
  L.p0_off = L.c_off + smax * smax * 4;
  L.p1_off = L.p0_off + 16 * smax * 4;
  L.y_off = L.p1_off + 16 * smax * 4;
  L.d_off = L.y_off + 16 * (h + 1) * 4;
  L.gi_off = L.d_off + 32 * 4;
  L.acc_off = L.gi_off + 16;
  L.total = L.acc_off + 4 * (kHafMaxPairs + 1) * 4;
  L.total = (L.total + 3) & ~3;  // 32-byte multiple
  return L;
}

__device__ __forceinline__ ddc ddc_zero() { return ddc{dd_make(0.0), dd_make(0.0)}; }

__device__ __forceinline__ ddc strip_pair_trace_dd(const double* X, const double* Y, int rows, int s,
                                                   int lane) {
  ddc acc = ddc_zero();
  const int tot = rows * s;
  for (int e = lane; e < tot; e += 32) {
    int i = e / s, t = e - i * s;
    acc = ddc_add(acc, ddc_mul(ld_ddc(X + (i * s + t) * 4), ld_ddc(Y + ((i ^ 1) * s + (t ^ 1)) * 4)));
  }
  return warp_sum_ddc(acc);
}

__device__ __forceinline__ void strip_matvec_dd(const double* P, const double* Dv, double* Y, int col,
                                                int hp1, int rows, int s, int lane) {
  const int i = lane >> 1, half = lane & 1;
  ddc acc = ddc_zero();
  if (i < rows)
    for (int t = half; t < s; t += 2) acc = ddc_add(acc, ddc_mul(ld_ddc(P + (i * s + t) * 4), ld_ddc(Dv + t * 4)));
  acc = ddc_add(acc, shfl_xor_ddc(acc, 1));
  if (half == 0 && i < 16) st_ddc(Y + (i * hp1 + col) * 4, i < rows ? acc : ddc_zero());
}

static __device__ ddc haf_subset_term_dd(const double* __restrict__ A, int N, int n, uint32_t mask, bool loop,
                                  double* ws, const HafDDLayout& Lw, int lane) {
  const int m = __popc(mask);
  if (m == 0) return ddc{dd_make(n == 0 ? 1.0 : 0.0), dd_make(0.0)};
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
  for (int e = lane; e < s * s; e += 32) {
    int r = e / s, c = e - r * s;
    int rr = gi[r], cc = gi[c ^ 1];
    cplx v = (loop || rr != cc) ? ld_c(A + ((size_t)rr * N + cc) * 2) : mkc(0.0, 0.0);
    st_ddc(Cs + e * 4, ddc_make(v));
  }
  if (loop && lane < s) st_ddc(Dv + lane * 4, ddc_make(ld_c(A + ((size_t)gi[lane] * N + gi[lane]) * 2)));
  for (int k = lane; k <= n; k += 32) {
    st_ddc(acc_p + 4 * k, ddc_zero());
    st_ddc(acc_v + 4 * k, ddc_zero());
  }
  __syncwarp();
  {
    ddc t = lane < s ? ld_ddc(Cs + (lane * s + lane) * 4) : ddc_zero();
    t = warp_sum_ddc(t);
    if (lane == 0) st_ddc(acc_p + 4, t);
  }
  const int nstrips = (s + 15) >> 4;
  for (int st = 0; st < nstrips; ++st) {
    const int r0 = st * 16;
    const int rows = min(16, s - r0);
    double* Pa = P0;
    double* Pb = P1;
    for (int e = lane; e < 16 * s; e += 32) {
      int i = e / s;
      st_ddc(Pa + e * 4, i < rows ? ld_ddc(Cs + ((r0 + i) * s + (e - i * s)) * 4) : ddc_zero());
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
            for (int t = 0; t < s; ++t) acc = ddc_add(acc, ddc_mul(ld_ddc(Pa + (i * s + t) * 4), ld_ddc(Cs + (t * s + j) * 4)));
            st_ddc(Pb + (i * s + j) * 4, acc);
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
  __syncwarp();
  ddc coeff = ld_ddc(ev + 4 * n);
  __syncwarp();
  return ((n - m) & 1) ? ddc_neg(coeff) : coeff;
}

}  // namespace gbsb
