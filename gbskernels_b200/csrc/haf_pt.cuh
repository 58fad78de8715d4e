// haf_pt.cuh -- hafnian and loop hafnian by the power-trace formula, one warp per
// subset, binary64 on the FP64 tensor cores (mma.sync .m16n8k8 / .m16n8k4 .f64).
//
// Algorithm (the reference's, cpu_ref/hafnian.py:101-129 and
// cpu_ref/loop_hafnian.py:65-108; device form core/hafnian.cu:41-133,
// core/loop_hafnian.cu:45-130):
//   haf(A) = sum_{S subset [n]} (-1)^(n-|S|) [lambda^n] exp( sum_k g_k lambda^k ),
//   C = B_S X  (B_S the principal submatrix on the pairs in S, X swaps each pair),
//   k g_k = tr(C^k)/2                      (ordinary hafnian, diagonal ignored)
//   k g_k = tr(C^k)/2 + k (1/2) d^T X C^{k-1} d   (loop hafnian, d = diag B_S),
//   [lambda^n] exp(.) by the Newton recurrence e_j = (1/j) sum_k (k g_k) e_{j-k}.
//
// B200 mapping (this repository's own design):
//   * One warp evaluates one subset at a time; C (s x s complex, s = 2|S|) is
//     staged in shared memory.
//   * The 16-row strips of C^a run their chains one after the other:
//     C^{a+1} = C^a C on the FP64 tensor cores through the real embedding
//     [Re P, Im P] (interleaved) x B', B'[2k+p][2j+q] = (p ? iC : C)[k][j] component
//     (q ? im : re): one m16n8k8 mma consumes four complex columns (an m16n8k4
//     finishes an odd count).
//   * Since C^T = X C X (B_S symmetric), (C^a)^T = X C^a X and
//       tr(C^{2a})   = sum_{i,t} C^a[i][t]     C^a[i^1][t^1]
//       tr(C^{2a-1}) = sum_{i,t} C^a[i][t] C^{a-1}[i^1][t^1],
//     so powers up to h = ceil(n/2) give every trace p_1..p_n: h-1 products per
//     subset instead of the reference's n-1.  In the mma accumulator layout the
//     partner element (i^1, t^1) of a lane's element sits in lane ^ 5, same
//     register; both traces read it from shared memory: the odd one from the
//     previous power before it is overwritten in place, the even one from the new
//     power once stored.
//   * The live column tiles of a subset are a prefix, so every tile loop leaves at
//     the first dead tile (one warp-uniform test per tile).
//   * Loop term: with y_a = C^a d, d^T X C^{a+b} d = (X y_a)^T y_b, so
//     v_k = (1/2) sum_i y_a[i^1] y_b[i] with a + b = k - 1 from the same powers.
#pragma once

#include "cert.cuh"
#include "gbs_common.cuh"

namespace gbsb {

constexpr int kHafMaxN = 32;                 // matrix side cap of the tensor-core path
constexpr int kHafMaxPairs = kHafMaxN / 2;   // n
constexpr int kHafMaxPow = (kHafMaxPairs + 1) / 2;  // h

// Strides (in complex elements) chosen for conflict-free fragment loads.
__host__ __device__ inline int haf_c_stride(int s) { return ((s + 3) / 8) * 8 + 4; }   // == 4 (mod 8)
// The power's row stride, per launch width (it changes no value): the 8-tile path
// (wide) takes == 4 (mod 8), conflict-free 16-byte stores and odd-trace loads; the
// 4-tile path == 2 (mod 4), conflict-free 8-byte A-fragment loads, which dominate
// its small subsets (measured: the wide choice gave the mixed queue +3 %, the narrow
// one config 1 +2.5 %).
__host__ __device__ inline int haf_p_stride(int s, bool wide) {
  return wide ? ((s + 3) / 8) * 8 + 4 : ((s % 4 == 2) ? s : s + 2);
}
__host__ __device__ inline int haf_strips(int s) { return (s + 15) / 16; }

// Per-warp shared-memory workspace (doubles), laid out for a launch-wide max s.
// The 16-row strips of a subset run their power chains one after the other, so
// the power and the loop vectors are held for one strip only.
// Batched Newton recurrence: the traces of kHafRing consecutive subsets are parked
// in a ring (slot: kg[1..n] and the sign, n <= smax / 2), then kHafRing lanes run
// one recurrence each.  Slot k[0] holds (sign, 0) or (0, 0) for an empty subset.
constexpr int kHafRing = 8;

struct HafLayout {
  int smax;
  int slot;  // complex entries per ring slot (smax / 2 + 1)
  int c_off, p_off, y_off, d_off, gi_off, acc_off, ring_off, total;  // in doubles
  // certified tier only: |C|, the bound-path power, row bounds, trace-bound sums,
  // the Newton coefficients
  int ca_off, m_off, ym_off, bt_off, ev_off;
  // certified tier: the ring of parked subsets' kg balls (cslot doubles per slot:
  // entry 0 = sign, halving flag; entries 1..n = re, im, radius)
  int cring_off, cslot;
};
__host__ __device__ inline HafLayout haf_layout(int smax, bool cert = false) {
  HafLayout L;
  if (smax < 2) smax = 2;
  L.smax = smax;
  const int cs = haf_c_stride(smax), ps = haf_p_stride(smax, smax > 16);
  const int rows = 16 * haf_strips(smax);
  const int h = (smax / 2 + 1) / 2;
  const int np1 = smax / 2 + 1;
  L.slot = np1;
  L.c_off = 0;
  L.p_off = L.c_off + rows * cs * 2;       // C, every strip (zero padding rows)
  L.y_off = L.p_off + 16 * ps * 2;         // the power of one strip
  L.d_off = L.y_off + 16 * (h + 1) * 2;    // the loop vectors of one strip
  L.gi_off = L.d_off + ((smax + 3) & ~3) * 2;  // d, zero-padded to whole column tiles
  L.acc_off = L.gi_off + ((smax + 3) / 4) * 2;  // smax ints, 16-byte multiple
  L.ring_off = L.acc_off + 2 * np1 * 2;    // acc_p, acc_v
  L.total = L.ring_off + kHafRing * np1 * 2;
  L.total = (L.total + 1) & ~1;  // 16-byte multiple
  L.ca_off = L.m_off = L.ym_off = L.bt_off = L.ev_off = L.cring_off = L.cslot = 0;
  if (cert) {
    L.ca_off = L.total;
    L.m_off = L.ca_off + rows * cs * 2;
    L.ym_off = L.m_off + rows * ps * 2;
    L.bt_off = L.ym_off + rows * (h + 1);
    L.ev_off = L.bt_off + 2 * (kHafMaxPairs + 2);
    L.total = L.ev_off + (kHafMaxPairs + 1) * 2;
    L.total = (L.total + 1) & ~1;
    L.cslot = (3 * np1 + 1) & ~1;
    L.cring_off = L.total;
    L.total = L.cring_off + kHafRing * L.cslot;
  }
  return L;
}

// Sum of four values over the warp, scattered: every lane gets the total of value
// 2 ((lane >> 4) & 1) + ((lane >> 3) & 1) (6 shuffles instead of 4 x 5).
__device__ __forceinline__ double warp_sum4_scatter(double v0, double v1, double v2, double v3, int lane) {
  const bool b4 = (lane & 16) != 0, b3 = (lane & 8) != 0;
  double k0 = b4 ? v2 : v0, k1 = b4 ? v3 : v1;
  k0 += shfl_xor_d(b4 ? v0 : v2, 16);
  k1 += shfl_xor_d(b4 ? v1 : v3, 16);
  double k = b3 ? k1 : k0;
  k += shfl_xor_d(b3 ? k0 : k1, 8);
  k += shfl_xor_d(k, 4);
  k += shfl_xor_d(k, 2);
  k += shfl_xor_d(k, 1);
  return k;
}

// ---------------------------------------------------------------------------
// D = P * C for every strip of P (rows 16 MS, complex), accumulators in the mma
// layout: D[ms][nt][0..3] = rows (16ms+g, 16ms+g+8), complex column 4nt+t4 (re, im).
template <int NT, int MS>
__device__ __forceinline__ void power_product(const double* __restrict__ P, const double* __restrict__ Cs, int s,
                                              int cs, int ps, int ntn, int lane, double (&D)[MS][NT][4]) {
  // P: the previous power (A operand, row stride ps complex); Cs: C (B' source, stride cs)
  // one accumulator chain per tile for every tile width: the 4- and 8-tile code paths
  // then give bit-identical results for the subsets both can run (s <= 16)
  constexpr int KS2 = 1;
  const int g = lane >> 2, t4 = lane & 3;
  double acc[KS2][MS][NT][4];
#pragma unroll
  for (int k2 = 0; k2 < KS2; ++k2)
#pragma unroll
    for (int ms = 0; ms < MS; ++ms)
#pragma unroll
      for (int nt = 0; nt < NT; ++nt)
        acc[k2][ms][nt][0] = acc[k2][ms][nt][1] = acc[k2][ms][nt][2] = acc[k2][ms][nt][3] = 0.0;
  // B' fragment of this lane: C[k][j] component (p ^ q), negated when p & !q, with
  // k = 2 ks + (t4 >> 1), p = t4 & 1, j = 4 nt + (g >> 1), q = g & 1.
  const double* bptr = Cs + ((t4 >> 1) * cs + (g >> 1)) * 2 + ((t4 ^ g) & 1);
  const unsigned long long sgn = ((t4 & 1) && !(g & 1)) ? 0x8000000000000000ull : 0ull;
  const double* ap = P + g * ps * 2 + t4;
  const int ksn = s >> 1;  // K = 2s real columns: ksn slices of 4, paired into m16n8k8 steps
  // k8 step j = k4 slices 2j (A columns t4, B' rows t4) and 2j + 1 (A columns t4 + 4,
  // B' rows t4 + 4)
  auto step8 = [&](int j, int k2) {
    const int k0 = 2 * j, k1 = 2 * j + 1;
    double a0[MS], a1[MS], a2[MS], a3[MS];
#pragma unroll
    for (int ms = 0; ms < MS; ++ms) {
      a0[ms] = ap[(16 * ms) * ps * 2 + 4 * k0];
      a1[ms] = ap[(16 * ms + 8) * ps * 2 + 4 * k0];
      a2[ms] = ap[(16 * ms) * ps * 2 + 4 * k1];
      a3[ms] = ap[(16 * ms + 8) * ps * 2 + 4 * k1];
    }
    const double* bp0 = bptr + k0 * 4 * cs;
    const double* bp1 = bptr + k1 * 4 * cs;
    // the live tiles are a prefix: one exit test per tile; the next live tile's
    // fragments are loaded before this tile's mma, so their latency overlaps it
    double nb0 = bp0[0], nb1 = bp1[0];
#pragma unroll
    for (int nt = 0; nt < NT; ++nt) {
      const double b0 = __longlong_as_double(__double_as_longlong(nb0) ^ sgn);
      const double b1 = __longlong_as_double(__double_as_longlong(nb1) ^ sgn);
      const bool more = nt + 1 < NT && nt + 1 < ntn;
      if (more) {
        nb0 = bp0[(nt + 1) * 8];
        nb1 = bp1[(nt + 1) * 8];
      }
#pragma unroll
      for (int ms = 0; ms < MS; ++ms) dmma_m16n8k8(acc[k2][ms][nt], a0[ms], a1[ms], a2[ms], a3[ms], b0, b1);
      if (!more) break;
    }
  };
  // a trailing single k4 slice when ksn is odd
  auto step4 = [&](int ks, int k2) {
    double a0[MS], a1[MS];
#pragma unroll
    for (int ms = 0; ms < MS; ++ms) {
      a0[ms] = ap[(16 * ms) * ps * 2 + 4 * ks];
      a1[ms] = ap[(16 * ms + 8) * ps * 2 + 4 * ks];
    }
    const double* bp = bptr + ks * 4 * cs;
#pragma unroll
    for (int nt = 0; nt < NT; ++nt) {
      if (nt > 0 && nt >= ntn) break;
      const double b = __longlong_as_double(__double_as_longlong(bp[nt * 8]) ^ sgn);
#pragma unroll
      for (int ms = 0; ms < MS; ++ms) dmma_m16n8k4(acc[k2][ms][nt], a0[ms], a1[ms], b);
    }
  };
  const int n8 = ksn >> 1;
  if constexpr (KS2 == 2) {
    int j = 0;
#pragma unroll 1
    for (; j + 1 < n8; j += 2) {
      step8(j, 0);
      step8(j + 1, 1);
    }
    if (j < n8) step8(j, 0);
    if (ksn & 1) step4(ksn - 1, 1);
#pragma unroll
    for (int ms = 0; ms < MS; ++ms)
#pragma unroll
      for (int nt = 0; nt < NT; ++nt)
#pragma unroll
        for (int q = 0; q < 4; ++q) D[ms][nt][q] = __dadd_rn(acc[0][ms][nt][q], acc[KS2 - 1][ms][nt][q]);
  } else {
#pragma unroll 1
    for (int j = 0; j < n8; ++j) step8(j, 0);
    if (ksn & 1) step4(ksn - 1, 0);
#pragma unroll
    for (int ms = 0; ms < MS; ++ms)
#pragma unroll
      for (int nt = 0; nt < NT; ++nt)
#pragma unroll
        for (int q = 0; q < 4; ++q) D[ms][nt][q] = acc[0][ms][nt][q];
  }
}

// Load P (power a, complex, stride ps) into the accumulator layout.
template <int NT, int MS>
__device__ __forceinline__ void load_acc(const double* P, int ps, int s, int lane, double (&D)[MS][NT][4]) {
  const int g = lane >> 2, t4 = lane & 3;
#pragma unroll
  for (int ms = 0; ms < MS; ++ms)
#pragma unroll
    for (int nt = 0; nt < NT; ++nt) {
      const int col = 4 * nt + t4;
      cplx x0 = mkc(0.0, 0.0), x1 = mkc(0.0, 0.0);
      if (col < s) {
        x0 = ld_c(P + ((16 * ms + g) * ps + col) * 2);
        x1 = ld_c(P + ((16 * ms + g + 8) * ps + col) * 2);
      }
      D[ms][nt][0] = x0.re; D[ms][nt][1] = x0.im; D[ms][nt][2] = x1.re; D[ms][nt][3] = x1.im;
    }
}

// Store the accumulators into P (rows < 16 MS, columns < s).
template <int NT, int MS>
__device__ __forceinline__ void store_acc(double* P, int ps, int s, int lane, const double (&D)[MS][NT][4]) {
  const int g = lane >> 2, t4 = lane & 3;
#pragma unroll
  for (int ms = 0; ms < MS; ++ms)
#pragma unroll
    for (int nt = 0; nt < NT; ++nt) {
      const int col = 4 * nt + t4;
      if (col < s) {
        st_c(P + ((16 * ms + g) * ps + col) * 2, mkc(D[ms][nt][0], D[ms][nt][1]));
        st_c(P + ((16 * ms + g + 8) * ps + col) * 2, mkc(D[ms][nt][2], D[ms][nt][3]));
      }
    }
}

// ---- one strip of a power in the binary64 value path.  The guards: LIVE (the 8-tile
// path) keeps every live tile's four columns, including the columns s..4 ntn - 1,
// which hold zeros wherever they are stored (the staged C, the powers, d); otherwise
// (the 4-tile path, whose power stride can be below 4 ntn) only the columns < s.
// The live tiles are a prefix, so a LIVE loop leaves at the first dead tile: one
// warp-uniform exit test per tile instead of a divergent branch per column.
template <int NT, bool LIVE>
__device__ __forceinline__ bool strip_col(int nt, int ntn, int col, int s, bool& stop) {
  stop = LIVE && nt > 0 && nt >= ntn;
  return LIVE || col < s;
}

// Load one strip (rows g / g + 8 of each tile, row stride ps complex) into the
// accumulator layout; tiles not loaded hold zeros.
template <int NT, bool LIVE>
__device__ __forceinline__ void load_strip(const double* P, int ps, int s, int ntn, int lane, double (&D)[1][NT][4]) {
  const int g = lane >> 2, t4 = lane & 3;
#pragma unroll
  for (int nt = 0; nt < NT; ++nt) D[0][nt][0] = D[0][nt][1] = D[0][nt][2] = D[0][nt][3] = 0.0;
#pragma unroll
  for (int nt = 0; nt < NT; ++nt) {
    const int col = 4 * nt + t4;
    bool stop;
    const bool use = strip_col<NT, LIVE>(nt, ntn, col, s, stop);
    if (stop) break;
    if (use) {
      const cplx x0 = ld_c(P + (g * ps + col) * 2), x1 = ld_c(P + ((g + 8) * ps + col) * 2);
      D[0][nt][0] = x0.re; D[0][nt][1] = x0.im; D[0][nt][2] = x1.re; D[0][nt][3] = x1.im;
    }
  }
}

template <int NT, bool LIVE>
__device__ __forceinline__ void store_strip(double* P, int ps, int s, int ntn, int lane, const double (&D)[1][NT][4]) {
  const int g = lane >> 2, t4 = lane & 3;
#pragma unroll
  for (int nt = 0; nt < NT; ++nt) {
    const int col = 4 * nt + t4;
    bool stop;
    const bool use = strip_col<NT, LIVE>(nt, ntn, col, s, stop);
    if (stop) break;
    if (use) {
      st_c(P + (g * ps + col) * 2, mkc(D[0][nt][0], D[0][nt][1]));
      st_c(P + ((g + 8) * ps + col) * 2, mkc(D[0][nt][2], D[0][nt][3]));
    }
  }
}

// Lane partial of sum_{i,t} D[i][t] * Q[i^1][t^1] (four independent accumulators:
// rows g / g + 8 x even / odd tiles).  Q = the previous power gives the odd trace
// tr(C^{2a-1}); Q = D itself, once stored, the even trace tr(C^{2a}) (the partner
// element is another lane's accumulator: reading it back from shared memory costs two
// loads per tile where exchanging it costs eight shuffles).
template <int NT, bool LIVE>
__device__ __forceinline__ cplx pair_partial(const double (&D)[1][NT][4], const double* Q, int ps, int s, int ntn,
                                             int lane) {
  const int g = lane >> 2, t4 = lane & 3;
  cplx acc[4] = {mkc(0.0, 0.0), mkc(0.0, 0.0), mkc(0.0, 0.0), mkc(0.0, 0.0)};
#pragma unroll
  for (int nt = 0; nt < NT; ++nt) {
    const int col = 4 * nt + t4;
    bool stop;
    const bool use = strip_col<NT, LIVE>(nt, ntn, col, s, stop);
    if (stop) break;
    if (use) {
      const int cp = col ^ 1;
      const cplx q0 = ld_c(Q + ((g ^ 1) * ps + cp) * 2);
      const cplx q1 = ld_c(Q + (((g + 8) ^ 1) * ps + cp) * 2);
      acc[2 * (nt & 1)] = cfma(mkc(D[0][nt][0], D[0][nt][1]), q0, acc[2 * (nt & 1)]);
      acc[2 * (nt & 1) + 1] = cfma(mkc(D[0][nt][2], D[0][nt][3]), q1, acc[2 * (nt & 1) + 1]);
    }
  }
  return cadd(cadd(acc[0], acc[1]), cadd(acc[2], acc[3]));
}

// y[row] = sum_t D[row][t] d[t] for the rows of this lane's group; lanes t4 == 0
// write Y[row * hp1 + col].
template <int NT, bool LIVE>
__device__ __forceinline__ void rows_times_d(const double (&D)[1][NT][4], const double* Dv, double* Y, int col,
                                             int hp1, int s, int ntn, int lane) {
  const int g = lane >> 2, t4 = lane & 3;
  cplx y0 = mkc(0.0, 0.0), y1 = mkc(0.0, 0.0);
#pragma unroll
  for (int nt = 0; nt < NT; ++nt) {
    const int c = 4 * nt + t4;
    bool stop;
    const bool use = strip_col<NT, LIVE>(nt, ntn, c, s, stop);
    if (stop) break;
    if (use) {
      const cplx dv = ld_c(Dv + c * 2);
      y0 = cfma(mkc(D[0][nt][0], D[0][nt][1]), dv, y0);
      y1 = cfma(mkc(D[0][nt][2], D[0][nt][3]), dv, y1);
    }
  }
#pragma unroll
  for (int m = 1; m <= 2; m <<= 1) {
    y0.re += shfl_xor_d(y0.re, m); y0.im += shfl_xor_d(y0.im, m);
    y1.re += shfl_xor_d(y1.re, m); y1.im += shfl_xor_d(y1.im, m);
  }
  if (t4 == 0) {
    st_c(Y + (g * hp1 + col) * 2, y0);
    st_c(Y + ((g + 8) * hp1 + col) * 2, y1);
  }
}

// ---- bound path helpers (certified tier): real parts only, upward rounding
template <int NT, int MS>
__device__ __forceinline__ double even_bound(const double (&D)[MS][NT][4]) {
  double acc = 0.0;
#pragma unroll
  for (int ms = 0; ms < MS; ++ms)
#pragma unroll
    for (int nt = 0; nt < NT; ++nt) {
      acc = ru_fma(D[ms][nt][0], shfl_xor_d(D[ms][nt][0], 5), acc);
      acc = ru_fma(D[ms][nt][2], shfl_xor_d(D[ms][nt][2], 5), acc);
    }
  return acc;
}
template <int NT, int MS>
__device__ __forceinline__ double odd_bound(const double (&D)[MS][NT][4], const double* Q, int ps, int s, int lane) {
  const int g = lane >> 2, t4 = lane & 3;
  double acc = 0.0;
#pragma unroll
  for (int ms = 0; ms < MS; ++ms)
#pragma unroll
    for (int nt = 0; nt < NT; ++nt) {
      const int col = 4 * nt + t4;
      if (col < s) {
        const int cp = col ^ 1;
        acc = ru_fma(D[ms][nt][0], Q[((16 * ms + (g ^ 1)) * ps + cp) * 2], acc);
        acc = ru_fma(D[ms][nt][2], Q[((16 * ms + ((g + 8) ^ 1)) * ps + cp) * 2], acc);
      }
    }
  return acc;
}
template <int NT, int MS>
__device__ __forceinline__ void rows_bound(const double (&D)[MS][NT][4], const double* Dv, double* Ym, int col,
                                           int hp1, int s, int lane) {
  const int g = lane >> 2, t4 = lane & 3;
#pragma unroll
  for (int ms = 0; ms < MS; ++ms) {
    double y0 = 0.0, y1 = 0.0;
#pragma unroll
    for (int nt = 0; nt < NT; ++nt) {
      const int c = 4 * nt + t4;
      if (c < s) {
        const double dv = ru_abs_c(ld_c(Dv + c * 2));
        y0 = ru_fma(D[ms][nt][0], dv, y0);
        y1 = ru_fma(D[ms][nt][2], dv, y1);
      }
    }
#pragma unroll
    for (int m = 1; m <= 2; m <<= 1) {
      y0 = ru_add(y0, shfl_xor_d(y0, m));
      y1 = ru_add(y1, shfl_xor_d(y1, m));
    }
    if (t4 == 0) {
      Ym[(16 * ms + g) * hp1 + col] = y0;
      Ym[(16 * ms + g + 8) * hp1 + col] = y1;
    }
  }
}

// ---------------------------------------------------------------------------
// Bound path of the certified tiers for the compile-time tile shape: the powers of
// |C| (Ca; the previous power kept in M) give the trace-bound sums
// bT[k] += sum_{i,t} M_a[i][t] M_b[i^1][t^1] and the row bounds Ym[row][a] =
// M_a |d| (upward rounded).  Dv holds d as binary64 complex (zero beyond s).
template <int NT, int MS>
__device__ __noinline__ void haf_bound_powers(const double* Ca, double* M, double* Ym, const double* Dv, double* bT,
                                              int s, int cs, int ps, int n, int h, bool loop, int lane) {
  const int ntn = (2 * s + 7) >> 3;  // column tiles in use (<= NT)
  const int hp1 = h + 1;
  double Dm[MS][NT][4];
  load_acc<NT, MS>(Ca, cs, s, lane, Dm);
  {
    double tb = warp_sum_ru(even_bound<NT, MS>(Dm));
    if (lane == 0 && 2 <= n) bT[2] = ru_add(bT[2], tb);
  }
  if (loop) rows_bound<NT, MS>(Dm, Dv, Ym, 1, hp1, s, lane);
  for (int a = 2; a <= h; ++a) {
    const double* Qm = (a == 2) ? Ca : M;
    const int qs = (a == 2) ? cs : ps;
    power_product<NT, MS>(Qm, Ca, s, cs, qs, ntn, lane, Dm);
    double bo = warp_sum_ru(odd_bound<NT, MS>(Dm, Qm, qs, s, lane));
    double be = warp_sum_ru(even_bound<NT, MS>(Dm));
    if (lane == 0) {
      if (2 * a - 1 <= n) bT[2 * a - 1] = ru_add(bT[2 * a - 1], bo);
      if (2 * a <= n) bT[2 * a] = ru_add(bT[2 * a], be);
    }
    __syncwarp();
    store_acc<NT, MS>(M, ps, s, lane, Dm);
    if (loop) rows_bound<NT, MS>(Dm, Dv, Ym, a, hp1, s, lane);
    __syncwarp();
  }
}

// ---------------------------------------------------------------------------
// Power loop of one subset for the compile-time tile width (NT column tiles of 8
// real columns): the 16-row strips run their chains C, C^2, ..., C^h one after the
// other (the rows of a power evolve independently and a trace pair (i, i^1) never
// crosses a strip), each with the strip's power in P and its loop vectors in Y.
// Traces go to acc_p[k], the loop terms v_k = 1/2 sum_i y_a[i^1] y_b[i] to acc_v[k],
// strip by strip in a fixed order.
template <int NT>
__device__ __noinline__ void haf_powers(const double* Cs, double* P, double* Y, const double* Dv, double* acc_p,
                                        double* acc_v, int s, int cs, int ps, int n, int h, bool loop, int lane) {
  const int ntn = (2 * s + 7) >> 3;  // column tiles in use (<= NT)
  const int hp1 = h + 1;
  const int strips = haf_strips(s);
  const int vq = (lane >> 3) & 3;          // the total this lane holds after warp_sum4_scatter
  const bool vlead = (lane & 7) == 0;
  constexpr bool LIVE = NT == 8;  // the 8-tile power stride holds every live tile's columns
  for (int ms = 0; ms < strips; ++ms) {
    const int r0 = 16 * ms;
    const double* Cstrip = Cs + r0 * cs * 2;
    double D[1][NT][4];
    if (loop && lane < 16) st_c(Y + (lane * hp1) * 2, r0 + lane < s ? ld_c(Dv + (r0 + lane) * 2) : mkc(0.0, 0.0));
    // power 1 (= the strip of C, read in place with stride cs): p_2 and y_1
    load_strip<NT, LIVE>(Cstrip, cs, s, ntn, lane, D);
    {
      const cplx t = pair_partial<NT, LIVE>(D, Cstrip, cs, s, ntn, lane);
      const double tot = warp_sum4_scatter(t.re, t.im, 0.0, 0.0, lane);
      if (vlead && vq < 2 && 2 <= n) acc_p[4 + vq] += tot;
    }
    if (loop) rows_times_d<NT, LIVE>(D, Dv, Y, 1, hp1, s, ntn, lane);
    for (int a = 2; a <= h; ++a) {
      // the previous power: the strip of C (stride cs) for a = 2, then P (stride ps), in place
      const double* Q = (a == 2) ? Cstrip : P;
      const int qs = (a == 2) ? cs : ps;
      power_product<NT, 1>(Q, Cs, s, cs, qs, ntn, lane, D);
      const cplx to = pair_partial<NT, LIVE>(D, Q, qs, s, ntn, lane);  // odd trace, before Q is overwritten
      __syncwarp();
      store_strip<NT, LIVE>(P, ps, s, ntn, lane, D);
      if (loop) rows_times_d<NT, LIVE>(D, Dv, Y, a, hp1, s, ntn, lane);
      __syncwarp();
      const cplx te = pair_partial<NT, LIVE>(D, P, ps, s, ntn, lane);  // even trace, from the stored power
      const double tot = warp_sum4_scatter(to.re, to.im, te.re, te.im, lane);
      if (vlead) {
        const int k = vq < 2 ? 2 * a - 1 : 2 * a;
        if (k <= n) acc_p[2 * k + (vq & 1)] += tot;
      }
    }
    if (loop) {
      // this strip's share of v_k (lane k - 1, rows in order)
      __syncwarp();
      if (lane < n) {
        const int k = lane + 1;
        const int aa = (k - 1) >> 1, bb = k - 1 - aa;
        const int nr = min(16, s - r0);
        cplx t = mkc(0.0, 0.0);
        for (int i = 0; i < nr; ++i) t = cadd(t, cmul(ld_c(Y + ((i ^ 1) * hp1 + aa) * 2), ld_c(Y + (i * hp1 + bb) * 2)));
        st_c(acc_v + 2 * k, cadd(ld_c(acc_v + 2 * k), cscale(t, 0.5)));
      }
      __syncwarp();
    }
  }
}

// ---------------------------------------------------------------------------
// Real inputs (every imaginary part zero).  B_S and C = B_S X are real, so the
// powers need none of the complex embedding: real m16n8k8 products with K = s (not
// 2s) over s columns (not 2s), a quarter of the mma work, and real traces.  The
// identities, the half-power schedule and the trace accumulators (acc_p, acc_v:
// real parts, imaginary parts zero) are those of the complex path.
//
// Real mma fragment layout (m16n8k8 .f64): A rows g / g+8, columns t4 / t4+4;
// B rows t4 / t4+4, column g; accumulator rows g / g+8, columns 2 t4 / 2 t4 + 1.
// The trace partner (i^1, t^1) of a lane's element (g, 2t4) is (g^1, 2t4+1): lane ^ 4,
// the other register of the pair.

// Row stride (doubles) of the real C and power: at least the K padding (a multiple
// of 8) and == 4 (mod 16), which spreads both fragment loads over the 16 8-byte
// bank pairs of a half warp (rows t4 or g step by 4 banks pairs).
__host__ __device__ inline int haf_r_stride(int s) {
  const int k = (s + 7) & ~7;
  return ((k + 11) / 16) * 16 + 4;
}
struct HafRealLayout {
  int rs;                                    // row stride (doubles)
  int c_off, p_off, y_off, d_off, total;     // in doubles, from the real scratch base
};
__host__ __device__ inline HafRealLayout haf_real_layout(int smax) {
  HafRealLayout L;
  if (smax < 2) smax = 2;
  L.rs = haf_r_stride(smax);
  const int rows = 16 * haf_strips(smax);
  const int h = (smax / 2 + 1) / 2;
  L.c_off = 0;
  L.p_off = rows * L.rs;                     // C (rows and columns zero-padded)
  L.y_off = L.p_off + 16 * L.rs;             // the power of one strip
  L.d_off = L.y_off + 16 * (h + 1);          // the loop vectors of one strip
  L.total = L.d_off + L.rs;                  // d (zero beyond s)
  L.total = (L.total + 1) & ~1;
  return L;
}

// D = P * C on the real tiles in use (ntr of up to NT tiles of 8 columns), K = s:
// s / 8 m16n8k8 steps, then an m16n8k4 step when s % 8 <= 4, or one more m16n8k8
// step over zero-padded columns when s % 8 == 6.
template <int NT>
__device__ __forceinline__ void power_product_real(const double* __restrict__ P, const double* __restrict__ Cr, int s,
                                                   int rs, int ntr, int lane, double (&D)[NT][4]) {
  const int g = lane >> 2, t4 = lane & 3;
#pragma unroll
  for (int nt = 0; nt < NT; ++nt) D[nt][0] = D[nt][1] = D[nt][2] = D[nt][3] = 0.0;
  const double* ap = P + g * rs + t4;
  const double* bp = Cr + t4 * rs + g;
  const int n8 = (s + 2) >> 3;  // s % 8 == 6 rounds up to one more k8 step
#pragma unroll 1
  for (int j = 0; j < n8; ++j) {
    const int k0 = 8 * j;
    const double a0 = ap[k0], a1 = ap[8 * rs + k0], a2 = ap[k0 + 4], a3 = ap[8 * rs + k0 + 4];
    const double* b0p = bp + k0 * rs;
    const double* b1p = bp + (k0 + 4) * rs;
#pragma unroll
    for (int nt = 0; nt < NT; ++nt)
      if (nt < ntr) dmma_m16n8k8(D[nt], a0, a1, a2, a3, b0p[8 * nt], b1p[8 * nt]);
  }
  if ((s & 7) != 0 && (s & 7) <= 4) {
    const int k0 = 8 * n8;
    const double a0 = ap[k0], a1 = ap[8 * rs + k0];
    const double* b0p = bp + k0 * rs;
#pragma unroll
    for (int nt = 0; nt < NT; ++nt)
      if (nt < ntr) dmma_m16n8k4(D[nt], a0, a1, b0p[8 * nt]);
  }
}

template <int NT>
__device__ __forceinline__ void load_acc_real(const double* P, int rs, int ntr, int lane, double (&D)[NT][4]) {
  const int g = lane >> 2, t4 = lane & 3;
#pragma unroll
  for (int nt = 0; nt < NT; ++nt) {
    cplx x0 = mkc(0.0, 0.0), x1 = mkc(0.0, 0.0);
    if (nt < ntr) {
      x0 = ld_c(P + g * rs + 8 * nt + 2 * t4);
      x1 = ld_c(P + (g + 8) * rs + 8 * nt + 2 * t4);
    }
    D[nt][0] = x0.re; D[nt][1] = x0.im; D[nt][2] = x1.re; D[nt][3] = x1.im;
  }
}

template <int NT>
__device__ __forceinline__ void store_acc_real(double* P, int rs, int ntr, int lane, const double (&D)[NT][4]) {
  const int g = lane >> 2, t4 = lane & 3;
#pragma unroll
  for (int nt = 0; nt < NT; ++nt)
    if (nt < ntr) {
      st_c(P + g * rs + 8 * nt + 2 * t4, mkc(D[nt][0], D[nt][1]));
      st_c(P + (g + 8) * rs + 8 * nt + 2 * t4, mkc(D[nt][2], D[nt][3]));
    }
}

// Lane partial of sum_{i,t} D[i][t] D[i^1][t^1] (partner: lane ^ 4, other register).
template <int NT>
__device__ __forceinline__ double even_partial_real(const double (&D)[NT][4], int ntr) {
  double e0 = 0.0, e1 = 0.0;
#pragma unroll
  for (int nt = 0; nt < NT; ++nt) {
    if (nt >= ntr) continue;
    const double p0 = shfl_xor_d(D[nt][0], 4), p1 = shfl_xor_d(D[nt][1], 4);
    const double p2 = shfl_xor_d(D[nt][2], 4), p3 = shfl_xor_d(D[nt][3], 4);
    e0 = fma(D[nt][0], p1, e0);
    e1 = fma(D[nt][1], p0, e1);
    e0 = fma(D[nt][2], p3, e0);
    e1 = fma(D[nt][3], p2, e1);
  }
  return e0 + e1;
}

// Lane partial of sum_{i,t} D[i][t] Q[i^1][t^1], Q the previous power (stride rs).
template <int NT>
__device__ __forceinline__ double odd_partial_real(const double (&D)[NT][4], const double* Q, int rs, int ntr,
                                                   int lane) {
  const int g = lane >> 2, t4 = lane & 3;
  double o0 = 0.0, o1 = 0.0;
#pragma unroll
  for (int nt = 0; nt < NT; ++nt) {
    if (nt >= ntr) continue;
    const cplx q0 = ld_c(Q + (g ^ 1) * rs + 8 * nt + 2 * t4);
    const cplx q1 = ld_c(Q + ((g + 8) ^ 1) * rs + 8 * nt + 2 * t4);
    o0 = fma(D[nt][0], q0.im, o0);
    o1 = fma(D[nt][1], q0.re, o1);
    o0 = fma(D[nt][2], q1.im, o0);
    o1 = fma(D[nt][3], q1.re, o1);
  }
  return o0 + o1;
}

// y[row] = sum_t D[row][t] d[t] for the rows of this lane's group; lanes t4 == 0
// write Y[row * hp1 + col].
template <int NT>
__device__ __forceinline__ void rows_times_d_real(const double (&D)[NT][4], const double* Dr, double* Y, int col,
                                                  int hp1, int ntr, int lane) {
  const int g = lane >> 2, t4 = lane & 3;
  double y0 = 0.0, y1 = 0.0;
#pragma unroll
  for (int nt = 0; nt < NT; ++nt) {
    if (nt >= ntr) continue;
    const cplx dv = ld_c(Dr + 8 * nt + 2 * t4);
    y0 = fma(D[nt][0], dv.re, y0);
    y0 = fma(D[nt][1], dv.im, y0);
    y1 = fma(D[nt][2], dv.re, y1);
    y1 = fma(D[nt][3], dv.im, y1);
  }
#pragma unroll
  for (int m = 1; m <= 2; m <<= 1) {
    y0 += shfl_xor_d(y0, m);
    y1 += shfl_xor_d(y1, m);
  }
  if (t4 == 0) {
    Y[g * hp1 + col] = y0;
    Y[(g + 8) * hp1 + col] = y1;
  }
}

// Sum of two values over the warp: lanes with (lane >> 4) & 1 == b get the total of
// value b (5 shuffles).
__device__ __forceinline__ double warp_sum2_scatter(double v0, double v1, int lane) {
  const bool b4 = (lane & 16) != 0;
  double k = b4 ? v1 : v0;
  k += shfl_xor_d(b4 ? v0 : v1, 16);
  k += shfl_xor_d(k, 8);
  k += shfl_xor_d(k, 4);
  k += shfl_xor_d(k, 2);
  k += shfl_xor_d(k, 1);
  return k;
}

// The power loop of one real subset: the 16-row strips run their chains in turn
// (as haf_powers); traces go to the real parts of acc_p[k], the loop terms to acc_v[k].
template <int NT>
__device__ __noinline__ void haf_powers_real(const double* Cr, double* P, double* Y, const double* Dr, double* acc_p,
                                             double* acc_v, int s, int rs, int n, int h, bool loop, int lane) {
  const int ntr = (s + 7) >> 3;  // real column tiles in use (<= NT)
  const int hp1 = h + 1;
  const int strips = haf_strips(s);
  const bool lead = (lane & 15) == 0;  // lane 0: the odd total, lane 16: the even total
  const int half = lane >> 4;
  for (int ms = 0; ms < strips; ++ms) {
    const int r0 = 16 * ms;
    const double* Cstrip = Cr + r0 * rs;
    double D[NT][4];
    if (loop && lane < 16) Y[lane * hp1] = r0 + lane < s ? Dr[r0 + lane] : 0.0;
    load_acc_real<NT>(Cstrip, rs, ntr, lane, D);
    {
      const double tot = warp_sum_d(even_partial_real<NT>(D, ntr));
      if (lane == 0 && 2 <= n) acc_p[4] += tot;
    }
    if (loop) rows_times_d_real<NT>(D, Dr, Y, 1, hp1, ntr, lane);
    for (int a = 2; a <= h; ++a) {
      const double* Q = (a == 2) ? Cstrip : P;
      power_product_real<NT>(Q, Cr, s, rs, ntr, lane, D);
      const double to = odd_partial_real<NT>(D, Q, rs, ntr, lane);
      const double te = even_partial_real<NT>(D, ntr);
      const double tot = warp_sum2_scatter(to, te, lane);
      if (lead) {
        const int k = half == 0 ? 2 * a - 1 : 2 * a;
        if (k <= n) acc_p[2 * k] += tot;
      }
      __syncwarp();
      store_acc_real<NT>(P, rs, ntr, lane, D);
      if (loop) rows_times_d_real<NT>(D, Dr, Y, a, hp1, ntr, lane);
      __syncwarp();
    }
    if (loop) {
      __syncwarp();
      if (lane < n) {
        const int k = lane + 1;
        const int aa = (k - 1) >> 1, bb = k - 1 - aa;
        const int nr = min(16, s - r0);
        double t = 0.0;
        for (int i = 0; i < nr; ++i) t = fma(Y[(i ^ 1) * hp1 + aa], Y[i * hp1 + bb], t);
        acc_v[2 * k] += 0.5 * t;
      }
      __syncwarp();
    }
  }
}

// Stage the real C = B_S X (symmetric part, rows and columns zero-padded to the
// tiles read) and d for a real subset into the real scratch (after the layout's
// own areas); the certified tier also gets |C| and d in the complex layout, which
// its bound path reads.  Returns this lane's "tiny halving" flag (see the complex
// staging in haf_subset_term_tc).
// Entry (r, c) of the real C = B_S X as the symmetric part (x + y) / 2; zero outside
// the s x s block and on the skipped diagonal of a plain hafnian.  `tiny` (certified
// tier) records a halving that could round absolutely.
template <bool CERT>
__device__ __forceinline__ double haf_real_entry(const double* __restrict__ A, int N, int s, bool loop,
                                                 const int* gi, int r, int c, bool& tiny) {
  if (r >= s || c >= s) return 0.0;
  const int rr = gi[r], cc = gi[c ^ 1];  // X swaps the columns within each pair
  if (!loop && rr == cc) return 0.0;
  const double x = A[((size_t)rr * N + cc) * 2], y = A[((size_t)cc * N + rr) * 2];
  if constexpr (CERT) {
    const double w = x + y;
    if (x != y && fabs(w) > 0.0 && fabs(w) < 4.450147717014403e-308) tiny = true;
  }
  return 0.5 * (x + y);
}

template <bool CERT>
__device__ __noinline__ bool haf_stage_real(const double* __restrict__ A, int N, int s, bool loop, const int* gi,
                                            int smax, double* ws, double* rb, int lane) {
  const HafRealLayout R = haf_real_layout(smax);
  double* Cr = rb + R.c_off;
  double* Dr = rb + R.d_off;
  const int rs = R.rs;
  const int rows = 16 * haf_strips(s);
  const int rcols = 8 * ((s + 7) >> 3);
  bool tiny = false;
  const int dr = 32 / rcols, dc = 32 - dr * rcols;  // (r, c) advance per 32 elements
  int r = lane / rcols, c = lane - (lane / rcols) * rcols;
  for (int e = lane; e < rows * rcols; e += 32, r += dr, c += dc) {
    if (c >= rcols) {
      c -= rcols;
      ++r;
    }
    Cr[r * rs + c] = haf_real_entry<CERT>(A, N, s, loop, gi, r, c, tiny);
  }
  if (loop)
    for (int k = lane; k < rs; k += 32) Dr[k] = k < s ? A[((size_t)gi[k] * N + gi[k]) * 2] : 0.0;
  if constexpr (CERT) {
    const int cs = haf_c_stride(s);
    const int ccols = (((2 * s + 7) >> 3) << 2);
    double* Ca = ws + haf_layout(smax, true).ca_off;
    const int dr2 = 32 / ccols, dc2 = 32 - dr2 * ccols;
    int r2 = lane / ccols, c2 = lane - (lane / ccols) * ccols;
    for (int e = lane; e < rows * ccols; e += 32, r2 += dr2, c2 += dc2) {
      if (c2 >= ccols) {
        c2 -= ccols;
        ++r2;
      }
      st_c(Ca + (r2 * cs + c2) * 2, mkc(fabs(haf_real_entry<CERT>(A, N, s, loop, gi, r2, c2, tiny)), 0.0));
    }
    if (loop && lane < s)
      st_c(ws + haf_layout(smax, true).d_off + lane * 2, mkc(A[((size_t)gi[lane] * N + gi[lane]) * 2], 0.0));
  }
  return tiny;
}

// ---------------------------------------------------------------------------
// Evaluate the signed power-trace term of one subset `mask` of instance A (N x N
// complex, row-major, N = 2n even).  Returns the same ball in every lane (radius 0
// unless CERT).  `loop` selects the loop hafnian; `ws` is this warp's workspace.
// Binary64 tiers (CERT false): kg[1..n] and the sign are parked in the ring slot
// `slot` (required) instead of running the Newton recurrence (haf_ring_flush runs
// it for a whole ring); the certified tier runs it in ball arithmetic here.
template <bool CERT, bool REAL = false>
static __device__ cball haf_subset_term_tc(const double* __restrict__ A, int N, int n, uint32_t mask,
                                           bool loop, double* ws, const HafLayout& Lw, int lane,
                                           double* slot = nullptr) {
  const int m = __popc(mask);
  if (m == 0) {
    if (slot && lane == 0) st_c(slot, mkc(0.0, 0.0));  // empty subset: term 0 (n >= 1)
    return cball{mkc(n == 0 ? 1.0 : 0.0, 0.0), 0.0};
  }
  const int s = 2 * m;
  const int cs = haf_c_stride(s), ps = haf_p_stride(s, Lw.smax > 16);
  const int h = (n + 1) / 2, hp1 = h + 1;
  const int rows = 16 * haf_strips(s);
  double* Cs = ws + Lw.c_off;
  double* P = ws + Lw.p_off;        // one strip of the power
  double* Y = ws + Lw.y_off;        // one strip of loop vectors: [16][h+1] complex
  double* Dv = ws + Lw.d_off;       // d[0..s)
  int* gi = reinterpret_cast<int*>(ws + Lw.gi_off);
  double* acc_p = ws + Lw.acc_off;  // p[0..n]
  double* acc_v = acc_p + Lw.slot * 2;
  double* Ca = ws + Lw.ca_off;
  double* M = ws + Lw.m_off;
  double* Ym = ws + Lw.ym_off;
  double* bT = ws + Lw.bt_off;                  // trace bound sums T[k]
  double* bV = bT + (kHafMaxPairs + 2);         // loop bound sums V[k]

  // ---- stage C = B_S X (rows padded to 16 per strip with zeros) and d
  if (lane < s) {
    uint32_t mm = mask;
    for (int u = 0; u < (lane >> 1); ++u) mm &= mm - 1;
    gi[lane] = 2 * (__ffs(mm) - 1) + (lane & 1);
  }
  __syncwarp();
  bool tiny_halving = false;  // certified tier: see the staging below
  if constexpr (REAL) {
    tiny_halving = haf_stage_real<CERT>(A, N, s, loop, gi, Lw.smax, ws, ws + Lw.total, lane);
  } else {
    const int ccols = (((2 * s + 7) >> 3) << 2);  // columns read by the n-tiles (>= s)
    // rows s..rows-1 stay zero: they are the padding rows of the power-2 A operand
    const int dr = 32 / ccols, dc = 32 - dr * ccols;  // (r, c) advance per 32 elements
    int r = lane / ccols, c = lane - (lane / ccols) * ccols;
    if constexpr (!CERT) {
      // without divergent branches: rows < s element by element (a padding column
      // loads a valid entry and stores zero), then the padding rows as zeros over the
      // whole row stride.  The symmetric part (A + A^T)/2 is staged: see below.
      for (int e = lane; e < s * ccols; e += 32, r += dr, c += dc) {
        const bool wrap = c >= ccols;
        c = wrap ? c - ccols : c;
        r = wrap ? r + 1 : r;
        const bool in = c < s;
        const int rr = gi[r], cc = gi[in ? (c ^ 1) : 0];  // X swaps the columns within each pair
        const cplx x = ld_c(A + ((size_t)rr * N + cc) * 2), y = ld_c(A + ((size_t)cc * N + rr) * 2);
        const cplx v = cscale(cadd(x, y), 0.5);
        st_c(Cs + (r * cs + c) * 2, (in && (loop || rr != cc)) ? v : mkc(0.0, 0.0));
      }
      for (int e = lane; e < (rows - s) * cs; e += 32) st_c(Cs + (s * cs + e) * 2, mkc(0.0, 0.0));
    } else
    for (int e = lane; e < rows * ccols; e += 32, r += dr, c += dc) {
      if (c >= ccols) {
        c -= ccols;
        ++r;
      }
      cplx v = mkc(0.0, 0.0);
      if (c < s && r < s) {
        const int rr = gi[r], cc = gi[c ^ 1];  // X swaps the columns within each pair
        if (loop || rr != cc) {
          // the symmetric part (A + A^T)/2, exact for a symmetric A: the half-power
          // identities need B_S symmetric, and the reference's n-1 products of the
          // raw entries agree with those of the symmetric part to second order in
          // the antisymmetric part
          const cplx x = ld_c(A + ((size_t)rr * N + cc) * 2), y = ld_c(A + ((size_t)cc * N + rr) * 2);
          v = cscale(cadd(x, y), 0.5);
          if constexpr (CERT) {
            // halving a sum below twice the smallest normal can round absolutely: no
            // certificate for such an entry (the relative input bound would not hold)
            const cplx w = cadd(x, y);
            if ((x.re != y.re || x.im != y.im) && fmin(fabs(w.re) > 0.0 ? fabs(w.re) : 1.0,
                                                       fabs(w.im) > 0.0 ? fabs(w.im) : 1.0) < 4.450147717014403e-308)
              tiny_halving = true;
          }
        }
      }
      st_c(Cs + (r * cs + c) * 2, v);
      if constexpr (CERT) st_c(Ca + (r * cs + c) * 2, mkc(ru_abs_c(v), 0.0));
    }
    if (loop && lane < s) st_c(Dv + lane * 2, ld_c(A + ((size_t)gi[lane] * N + gi[lane]) * 2));
    else if (loop && lane < ((s + 3) & ~3)) st_c(Dv + lane * 2, mkc(0.0, 0.0));  // whole column tiles
  }
  for (int k = lane; k <= n; k += 32) {
    st_c(acc_p + 2 * k, mkc(0.0, 0.0));
    st_c(acc_v + 2 * k, mkc(0.0, 0.0));
    if constexpr (CERT) { bT[k] = 0.0; bV[k] = 0.0; }
  }
  __syncwarp();
  if constexpr (CERT) {
    if (loop && lane < rows) Ym[lane * hp1] = lane < s ? ru_abs_c(ld_c(Dv + lane * 2)) : 0.0;
  }
  // p_1 = tr(C)
  if constexpr (REAL) {
    const HafRealLayout R = haf_real_layout(Lw.smax);
    const double* Cr = ws + Lw.total + R.c_off;
    const double d = lane < s ? Cr[lane * R.rs + lane] : 0.0;
    const double t = warp_sum_d(d);
    if (lane == 0) st_c(acc_p + 2, mkc(t, 0.0));
    if constexpr (CERT) {
      const double a1 = warp_sum_ru(fabs(d));
      if (lane == 0) bT[1] = a1;
    }
  } else {
    cplx t = mkc(0.0, 0.0);
    if (lane < s) t = ld_c(Cs + (lane * cs + lane) * 2);
    t = warp_sum_c(t);
    if (lane == 0) st_c(acc_p + 2, t);
    if constexpr (CERT) {
      double a1 = lane < s ? ru_abs_c(ld_c(Cs + (lane * cs + lane) * 2)) : 0.0;
      a1 = warp_sum_ru(a1);
      if (lane == 0) bT[1] = a1;
    }
  }
  __syncwarp();

  // ONE tile width per launch: up to 4 column tiles when every matrix of the launch
  // has N <= 16 (every subset fits one strip), otherwise up to 8 for every subset
  // (unused tiles skipped at run time; s > 16 runs two strips in turn).  A single
  // hot code path keeps the instruction footprint within the instruction cache:
  // mixing the two widths in one launch measured slower (instruction-fetch stalls
  // 2.2 against 0.3 cycles per issue).  Both widths run the same operations on the
  // tiles in use, so a value does not depend on the launch it is part of.
  // A real subset runs its own loop (real tiles of 8 columns: up to 2 for N <= 16,
  // 4 above) on the real scratch.
  if constexpr (REAL) {
    const HafRealLayout R = haf_real_layout(Lw.smax);
    double* rb = ws + Lw.total;
    if (Lw.smax <= 16)
      haf_powers_real<2>(rb + R.c_off, rb + R.p_off, rb + R.y_off, rb + R.d_off, acc_p, acc_v, s, R.rs, n, h, loop,
                         lane);
    else
      haf_powers_real<4>(rb + R.c_off, rb + R.p_off, rb + R.y_off, rb + R.d_off, acc_p, acc_v, s, R.rs, n, h, loop,
                         lane);
  } else {
    if (Lw.smax <= 16) haf_powers<4>(Cs, P, Y, Dv, acc_p, acc_v, s, cs, ps, n, h, loop, lane);
    else haf_powers<8>(Cs, P, Y, Dv, acc_p, acc_v, s, cs, ps, n, h, loop, lane);
  }
  if constexpr (CERT) {
    __syncwarp();
    if (s <= 16) haf_bound_powers<4, 1>(Ca, M, Ym, Dv, bT, s, cs, ps, n, h, loop, lane);
    else haf_bound_powers<8, 2>(Ca, M, Ym, Dv, bT, s, cs, ps, n, h, loop, lane);
  }
  __syncwarp();

  if constexpr (CERT) {
    // loop bound sums V[k] = sum_i Ym[i^1][a] Ym[i][b] (the values v_k came with the powers)
    if (loop) {
      for (int k = 1; k <= n; ++k) {
        const int aa = (k - 1) >> 1, bb = k - 1 - aa;
        double vb = lane < s ? ru_mul(Ym[(lane ^ 1) * hp1 + aa], Ym[lane * hp1 + bb]) : 0.0;
        vb = warp_sum_ru(vb);
        if (lane == 0) bV[k] = vb;
      }
      __syncwarp();
    }
  }

  // ---- Newton recurrence (certified: lane 0, then broadcast through shared memory;
  // binary64 tiers: kg_k parked by lane k, the recurrence runs in haf_ring_flush)
  bool tiny_any = false;  // certified tier: a halving anywhere refuses the certificate
  if constexpr (CERT) tiny_any = __any_sync(0xffffffffu, tiny_halving);
  if (!CERT || lane == 0) {
    if constexpr (CERT) {
      // value-path coefficients: E_a <= c_a M_a with M_a = |C|^a, M_a <= phi_a M^_a
      const double g2s = gamma_ru((double)(2 * s), 2.0 * kU);  // FP64 MMA, faithful rounding
      const double sq2 = 1.4142135623730952;
      const double g64 = ru_mul(sq2, gamma_ru(64.0, kU));
      const double gy = ru_mul(sq2, gamma_ru((double)(s + 4), kU));
      // loop term: complex products (4u) summed sequentially over the rows of each
      // strip, then the strips (at most s + 1 sums; sqrt(2) gamma_{s+4} <= gamma_{2s+8}
      // per component pair)
      const double gv = ru_add(4.0 * kU, gamma_ru(2.0 * s + 8.0, kU));
      // Input error: the staged C^ is the rounded symmetric part, |C - C^| <= c1 |C^|
      // with c1 = u/(1-u) (exactly 0 for a symmetric A; charged regardless), so
      // |C^a| <= t_a M_a with t_a = (1 + c1)^a, and the power errors E_a <= c_a M_a
      // follow c_1 = c1, c_{a+1} = c_a + c1 t_a + sqrt2 gamma_2s (t_a + c_a).
      const double c1 = kUc;
      double ca[kHafMaxPow + 2], ph[kHafMaxPow + 2], ka[kHafMaxPow + 2], ta[kHafMaxPow + 2];
      ca[0] = 0.0; ph[0] = 1.0; ca[1] = c1; ph[1] = 1.0; ta[0] = 1.0; ta[1] = ru_add(1.0, c1);
      for (int a = 1; a <= h; ++a) {
        ca[a + 1] = ru_add(ru_add(ca[a], ru_mul(c1, ta[a])), ru_mul(ru_mul(sq2, g2s), ru_add(ta[a], ca[a])));
        ph[a + 1] = ru_div(ph[a], rd_sub(1.0, g2s));
        ta[a + 1] = ru_mul(ta[a], ru_add(1.0, c1));
      }
      ka[0] = 0.0;
      for (int a = 1; a <= h; ++a) ka[a] = ru_add(ca[a], ru_mul(gy, ru_add(ta[a], ca[a])));
      cball kgb[kHafMaxPairs + 1];
      for (int k = 1; k <= n; ++k) {
        double ep;
        if (k == 1) {
          ep = ru_mul(ru_add(gamma_ru(6.0, kU), c1), bT[1]);
        } else if ((k & 1) == 0) {
          const int a = k / 2;
          double f = ru_add(ru_mul(ca[a], ru_add(ru_mul(2.0, ta[a]), ca[a])),
                            ru_mul(g64, ru_mul(ru_add(ta[a], ca[a]), ru_add(ta[a], ca[a]))));
          ep = ru_mul(ru_mul(f, ru_mul(ph[a], ph[a])), bT[k]);
        } else {
          const int a = (k + 1) / 2;
          double f = ru_add(ru_add(ru_add(ru_mul(ca[a], ta[a - 1]), ru_mul(ca[a - 1], ta[a])),
                                   ru_mul(ca[a], ca[a - 1])),
                            ru_mul(g64, ru_mul(ru_add(ta[a], ca[a]), ru_add(ta[a - 1], ca[a - 1]))));
          ep = ru_mul(ru_mul(f, ru_mul(ph[a], ph[a - 1])), bT[k]);
        }
        cball g{cscale(ld_c(acc_p + 2 * k), 0.5), ru_mul(0.5, ep)};
        if (loop) {
          const int aa = (k - 1) >> 1, bb = k - 1 - aa;
          double f = ru_add(ru_add(ru_add(ru_mul(ka[aa], ta[bb]), ru_mul(ka[bb], ta[aa])), ru_mul(ka[aa], ka[bb])),
                            ru_mul(gv, ru_mul(ru_add(ta[aa], ka[aa]), ru_add(ta[bb], ka[bb]))));
          double evb = ru_mul(0.5, ru_mul(ru_mul(f, ru_mul(ph[aa], ph[bb])), bV[k]));
          g = cb_add(g, cb_scale(cball{ld_c(acc_v + 2 * k), evb}, (double)k));
        }
        kgb[k] = g;
      }
      // parked for the recurrence (haf_ring_flush_cert: one lane per subset)
      slot[0] = ((n - m) & 1) ? -1.0 : 1.0;
      slot[1] = tiny_any ? 1.0 : 0.0;
      for (int k = 1; k <= n; ++k) {
        slot[3 * k] = kgb[k].z.re;
        slot[3 * k + 1] = kgb[k].z.im;
        slot[3 * k + 2] = kgb[k].r;
      }
    } else {
      if (lane == 0) st_c(slot, mkc(((n - m) & 1) ? -1.0 : 1.0, 0.0));
      if (lane >= 1 && lane <= n) {
        const int k = lane;
        cplx g = cscale(ld_c(acc_p + 2 * k), 0.5);
        if (loop) g = cadd(g, cscale(ld_c(acc_v + 2 * k), (double)k));
        st_c(slot + 2 * k, g);
      }
    }
  }
  __syncwarp();
  if constexpr (!CERT) {
    return cball{mkc(0.0, 0.0), 0.0};
  } else {
    return cball{mkc(0.0, 0.0), 0.0};  // the term comes from haf_ring_flush_cert
  }
}

// Certified tier: the Newton recurrences of `cnt` parked subsets in ball arithmetic,
// one lane each -- the operations of the one-subset recurrence, in its order, with
// e_j interleaved in the idle power buffer `e` (3 doubles per ball) -- and the ball
// sum of their signed terms over the lanes (warp_sum_cb, the grouping of the
// binary64 ring, so the value is the fp64 value bit for bit).  A subset with a
// halving that could round absolutely gets an infinite radius.
__device__ __forceinline__ cball haf_ring_flush_cert(const double* ring, int slotw, int cnt, int n, int lane,
                                                     double* e) {
  cball b{mkc(0.0, 0.0), 0.0};
  if (lane < cnt) {
    const double* sl = ring + lane * slotw;
    const double sign = sl[0];
    if (sign != 0.0) {
      double* el = e + lane * 3;
      constexpr int es = kHafRing * 3;  // doubles between e_j and e_{j+1} of a lane
      el[0] = 1.0;
      el[1] = 0.0;
      el[2] = 0.0;
      for (int j = 1; j <= n; ++j) {
        cball acc{mkc(0.0, 0.0), 0.0};
        for (int k = 1; k <= j; ++k) {
          const double* ek = el + (j - k) * es;
          acc = cb_add(acc, cb_mul(cball{mkc(sl[3 * k], sl[3 * k + 1]), sl[3 * k + 2]}, cball{mkc(ek[0], ek[1]), ek[2]}));
        }
        const cball ej = cb_div_int(acc, (double)j);
        double* ed = el + j * es;
        ed[0] = ej.z.re;
        ed[1] = ej.z.im;
        ed[2] = ej.r;
      }
      const double* en = el + n * es;
      const cplx coeff = mkc(en[0], en[1]);
      b = cball{sign < 0.0 ? cneg(coeff) : coeff, sl[1] != 0.0 ? INFINITY : en[2]};
    }
  }
  return warp_sum_cb(b);
}

// Run the Newton recurrence of `cnt` parked subsets, one lane each, and return
// the sum of their signed terms (every lane gets it; fixed butterfly order) and,
// in *absacc, the sum of |term|.  The coefficients e_0..e_n of lane l live in
// shared memory at e + (j kHafRing + l) complex entries (`e`: (n + 1) kHafRing
// complex entries that are free while the ring is flushed, the power buffer): a
// per-thread array would sit in local memory, whose stacks (8.7 KB per warp)
// overflow the L1 left beside the shared-memory workspaces.
__device__ __forceinline__ cplx haf_ring_flush(const double* ring, int slotw, int cnt, int n, int lane,
                                               double* absacc, double* e) {
  cplx term = mkc(0.0, 0.0);
  if (lane < cnt) {
    const double* sl = ring + lane * slotw * 2;
    const double sign = sl[0];
    if (sign != 0.0) {
      double* el = e + lane * 2;
      constexpr int es = kHafRing * 2;  // doubles between e_j and e_{j+1} of a lane
      st_c(el, mkc(1.0, 0.0));
      for (int j = 1; j <= n; ++j) {
        cplx acc = mkc(0.0, 0.0);
        for (int k = 1; k <= j; ++k) acc = cadd(acc, cmul(ld_c(sl + 2 * k), ld_c(el + (j - k) * es)));
        st_c(el + j * es, mkc(acc.re / j, acc.im / j));
      }
      term = cscale(ld_c(el + n * es), sign);
    }
  }
  if (absacc) *absacc = warp_sum_d(cabs_fast(term));
  return warp_sum_c(term);
}

}  // namespace gbsb
