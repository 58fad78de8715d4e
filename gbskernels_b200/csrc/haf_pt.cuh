// haf_pt.cuh -- hafnian and loop hafnian by the power-trace formula, one warp per
// subset, binary64 on the FP64 tensor cores (mma.sync .m16n8k4 .f64).
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
//   * Row strips of 16 rows evolve independently: strip(C^{a+1}) = strip(C^a) C.
//     The complex product runs on the FP64 tensor cores through the real
//     embedding  [Re P, Im P] (interleaved) x B',  B'[2k+p][2j+q] = (p ? iC : C)[k][j]
//     component (q ? im : re), so one m16n8k4 mma consumes two complex columns.
//   * Since C^T = X C X (B_S symmetric), (C^a)^T = X C^a X and
//       tr(C^{2a})   = sum_{i,t} C^a[i][t]     C^a[i^1][t^1]
//       tr(C^{2a-1}) = sum_{i,t} C^a[i][t] C^{a-1}[i^1][t^1],
//     so powers up to h = ceil(n/2) give every trace p_1..p_n: h-1 products per
//     subset instead of the reference's n-1.  Rows i and i^1 share a strip.
//   * Loop term: with y_a = C^a d, d^T X C^{a+b} d = (X y_a)^T y_b, so
//     v_k = (1/2) sum_i y_a[i^1] y_b[i] with a + b = k - 1 from the same powers.
#pragma once

#include "gbs_common.cuh"

namespace gbsb {

constexpr int kHafMaxN = 32;                 // matrix side cap of the tensor-core path
constexpr int kHafMaxPairs = kHafMaxN / 2;   // n
constexpr int kHafMaxPow = (kHafMaxPairs + 1) / 2;  // h

// Strides (in complex elements) chosen for conflict-free fragment loads.
__host__ __device__ inline int haf_c_stride(int s) { return ((s + 3) / 8) * 8 + 4; }   // == 4 (mod 8)
__host__ __device__ inline int haf_p_stride(int s) { return (s % 4 == 2) ? s : s + 2; }  // == 2 (mod 4)

// Per-warp shared-memory workspace (doubles), laid out for a launch-wide max s.
struct HafLayout {
  int smax;
  int c_off, p0_off, p1_off, y_off, d_off, gi_off, acc_off, total;  // in doubles
};
__host__ __device__ inline HafLayout haf_layout(int smax) {
  HafLayout L;
  if (smax < 2) smax = 2;
  L.smax = smax;
  int cs = haf_c_stride(smax), ps = haf_p_stride(smax);
  int h = (smax / 2 + 1) / 2;
  L.c_off = 0;
  L.p0_off = L.c_off + smax * cs * 2;
  L.p1_off = L.p0_off + 16 * ps * 2;
  L.y_off = L.p1_off + 16 * ps * 2;
  L.d_off = L.y_off + 16 * (h + 1) * 2;
  L.gi_off = L.d_off + 32 * 2;   // 32 ints
  L.acc_off = L.gi_off + 16;
  // acc: p[0..n], v[0..n], kg/e scratch [0..n] x 2  -> 4 * (kHafMaxPairs+1) complex
  L.total = L.acc_off + 4 * (kHafMaxPairs + 1) * 2;
  L.total = (L.total + 1) & ~1;  // 16-byte multiple
  return L;
}

// ---------------------------------------------------------------------------
// One strip product  P1[0:16][0:s] = P0[0:16][0:s] * C   (complex), NT n-tiles.
template <int NT>
__device__ __forceinline__ void strip_product(const double* __restrict__ P0, double* __restrict__ P1,
                                              const double* __restrict__ Cs, int s, int cs, int ps,
                                              int lane) {
  const int g = lane >> 2, t4 = lane & 3;
  double d[NT][4];
#pragma unroll
  for (int nt = 0; nt < NT; ++nt) d[nt][0] = d[nt][1] = d[nt][2] = d[nt][3] = 0.0;
  // B' fragment address for this lane: C[k][j] component (p ^ q), negated when p & !q,
  // with k = 2 ks + (t4 >> 1), p = t4 & 1, j = 4 nt + (g >> 1), q = g & 1.
  const double* bptr = Cs + ((t4 >> 1) * cs + (g >> 1)) * 2 + ((t4 ^ g) & 1);
  const unsigned long long sgn = ((t4 & 1) && !(g & 1)) ? 0x8000000000000000ull : 0ull;
  const double* a0p = P0 + g * ps * 2 + t4;
  const double* a1p = P0 + (g + 8) * ps * 2 + t4;
  const int ks_n = s >> 1;  // K = 2s real columns, 4 per slice
#pragma unroll 2
  for (int ks = 0; ks < ks_n; ++ks) {
    const double a0 = a0p[4 * ks];
    const double a1 = a1p[4 * ks];
    const double* bp = bptr + ks * 4 * cs;
#pragma unroll
    for (int nt = 0; nt < NT; ++nt) {
      double b = __longlong_as_double(__double_as_longlong(bp[nt * 8]) ^ sgn);
      dmma_m16n8k4(d[nt], a0, a1, b);
    }
  }
#pragma unroll
  for (int nt = 0; nt < NT; ++nt) {
    const int col = 4 * nt + t4;  // complex column held by this lane
    if (col < s) {
      double2* r0 = reinterpret_cast<double2*>(P1 + (g * ps + col) * 2);
      double2* r1 = reinterpret_cast<double2*>(P1 + ((g + 8) * ps + col) * 2);
      *r0 = make_double2(d[nt][0], d[nt][1]);
      *r1 = make_double2(d[nt][2], d[nt][3]);
    }
  }
}

__device__ __forceinline__ void strip_product_dispatch(const double* P0, double* P1, const double* Cs,
                                                       int s, int cs, int ps, int lane) {
  switch ((2 * s + 7) >> 3) {
    case 1: strip_product<1>(P0, P1, Cs, s, cs, ps, lane); break;
    case 2: strip_product<2>(P0, P1, Cs, s, cs, ps, lane); break;
    case 3: strip_product<3>(P0, P1, Cs, s, cs, ps, lane); break;
    case 4: strip_product<4>(P0, P1, Cs, s, cs, ps, lane); break;
    case 5: strip_product<5>(P0, P1, Cs, s, cs, ps, lane); break;
    case 6: strip_product<6>(P0, P1, Cs, s, cs, ps, lane); break;
    case 7: strip_product<7>(P0, P1, Cs, s, cs, ps, lane); break;
    default: strip_product<8>(P0, P1, Cs, s, cs, ps, lane); break;
  }
}


// sum over the strip's valid rows i and columns t of X[i][t] * Y[i^1][t^1].
__device__ __forceinline__ cplx strip_pair_trace(const double* X, const double* Y, int rows, int s,
                                                 int ps, int lane) {
  cplx acc = mkc(0.0, 0.0);
  const int tot = rows * s;
  for (int e = lane; e < tot; e += 32) {
    int i = e / s, t = e - i * s;
    acc = cfma(ld_c(X + (i * ps + t) * 2), ld_c(Y + ((i ^ 1) * ps + (t ^ 1)) * 2), acc);
  }
  return warp_sum_c(acc);
}

// Loop-term vectors y[i] = sum_t P[i][t] d[t] for the strip rows (lanes 2i, 2i+1 split t).
__device__ __forceinline__ void strip_matvec(const double* P, const double* dv, double* y, int rows,
                                             int s, int ps, int lane) {
  const int i = lane >> 1, half = lane & 1;
  cplx acc = mkc(0.0, 0.0);
  if (i < rows) {
    for (int t = half; t < s; t += 2) acc = cfma(ld_c(P + (i * ps + t) * 2), ld_c(dv + t * 2), acc);
  }
  acc.re += shfl_xor_d(acc.re, 1);
  acc.im += shfl_xor_d(acc.im, 1);
  if (half == 0 && i < 16) st_c(y + i * 2, i < rows ? acc : mkc(0.0, 0.0));
}

// ---------------------------------------------------------------------------
// Evaluate the signed power-trace term of one subset `mask` of instance A (N x N
// complex, row-major, N = 2n even).  Returns the same value in every lane.
// `loop` selects the loop hafnian.  `ws` is this warp's shared workspace.
static __device__ cplx haf_subset_term_tc(const double* __restrict__ A, int N, int n, uint32_t mask,
                                   bool loop, double* ws, const HafLayout& Lw, int lane) {
  const int m = __popc(mask);
  if (m == 0) return mkc(n == 0 ? 1.0 : 0.0, 0.0);
  const int s = 2 * m;
  const int cs = haf_c_stride(s), ps = haf_p_stride(s);
  const int h = (n + 1) / 2;
  double* Cs = ws + Lw.c_off;
  double* P0 = ws + Lw.p0_off;
  double* P1 = ws + Lw.p1_off;
  double* Y = ws + Lw.y_off;        // [16 rows][h+1] complex, row-major by power
  double* Dv = ws + Lw.d_off;       // d[0..s)
  double* acc_p = ws + Lw.acc_off;  // p[0..n]
  double* acc_v = acc_p + (kHafMaxPairs + 1) * 2;
  double* kg = acc_v + (kHafMaxPairs + 1) * 2;
  double* ev = kg + (kHafMaxPairs + 1) * 2;

  // ---- stage C = B_S X (and d) in shared memory.  gi[r] = global row of local row r.
  int* gi = reinterpret_cast<int*>(ws + Lw.gi_off);
  if (lane < s) {
    // position of the (lane/2)-th set bit of mask
    uint32_t mm = mask;
    for (int u = 0; u < (lane >> 1); ++u) mm &= mm - 1;
    gi[lane] = 2 * (__ffs(mm) - 1) + (lane & 1);
  }
  __syncwarp();
  const int ccols = (((2 * s + 7) >> 3) << 2);  // columns read by the n-tiles (>= s)
  for (int e = lane; e < s * ccols; e += 32) {
    int r = e / ccols, c = e - r * ccols;
    cplx v = mkc(0.0, 0.0);
    if (c < s) {
      int rr = gi[r], cc = gi[c ^ 1];  // X swaps the columns within each pair
      if (loop || rr != cc) v = ld_c(A + ((size_t)rr * N + cc) * 2);
    }
    st_c(Cs + (r * cs + c) * 2, v);
  }
  if (loop && lane < s) {
    int rr = gi[lane];
    st_c(Dv + lane * 2, ld_c(A + ((size_t)rr * N + rr) * 2));
  }
  for (int k = lane; k <= n; k += 32) {
    st_c(acc_p + 2 * k, mkc(0.0, 0.0));
    st_c(acc_v + 2 * k, mkc(0.0, 0.0));
  }
  __syncwarp();

  // p_1 = tr(C)
  {
    cplx t = mkc(0.0, 0.0);
    if (lane < s) t = ld_c(Cs + (lane * cs + lane) * 2);
    t = warp_sum_c(t);
    if (lane == 0) st_c(acc_p + 2, t);
  }

  const int nstrips = (s + 15) >> 4;
  for (int st = 0; st < nstrips; ++st) {
    const int r0 = st * 16;
    const int rows = min(16, s - r0);
    double* Pa = P0;  // power a-1 (after swap: current)
    double* Pb = P1;
    // P0 <- C rows of the strip (rows beyond s zero; both buffers zero-padded)
    for (int e = lane; e < 16 * ps; e += 32) {
      int i = e / ps, t = e - i * ps;
      cplx v = (i < rows && t < s) ? ld_c(Cs + ((r0 + i) * cs + t) * 2) : mkc(0.0, 0.0);
      st_c(Pa + e * 2, v);
      st_c(Pb + e * 2, mkc(0.0, 0.0));
    }
    __syncwarp();
    // power 1: p_2 = self trace; loop: y_0 = d, y_1 = C d
    {
      cplx t = strip_pair_trace(Pa, Pa, rows, s, ps, lane);
      if (lane == 0 && 2 <= n) st_c(acc_p + 4, cadd(ld_c(acc_p + 4), t));
    }
    if (loop) {
      if (lane < 16) st_c(Y + (lane * (h + 1) + 0) * 2, lane < rows ? ld_c(Dv + (r0 + lane) * 2) : mkc(0.0, 0.0));
      // y_1 rows -> Y[i][1]
      {
        const int i = lane >> 1, half = lane & 1;
        cplx acc = mkc(0.0, 0.0);
        if (i < rows)
          for (int t = half; t < s; t += 2) acc = cfma(ld_c(Pa + (i * ps + t) * 2), ld_c(Dv + t * 2), acc);
        acc.re += shfl_xor_d(acc.re, 1);
        acc.im += shfl_xor_d(acc.im, 1);
        if (half == 0 && i < 16) st_c(Y + (i * (h + 1) + 1) * 2, i < rows ? acc : mkc(0.0, 0.0));
      }
    }
    __syncwarp();
    for (int a = 2; a <= h; ++a) {
      strip_product_dispatch(Pa, Pb, Cs, s, cs, ps, lane);
      __syncwarp();
      // p_{2a-1} = tr(C^a C^{a-1}),  p_{2a} = tr(C^a C^a)
      cplx todd = strip_pair_trace(Pb, Pa, rows, s, ps, lane);
      cplx tev = strip_pair_trace(Pb, Pb, rows, s, ps, lane);
      if (lane == 0) {
        if (2 * a - 1 <= n) st_c(acc_p + 2 * (2 * a - 1), cadd(ld_c(acc_p + 2 * (2 * a - 1)), todd));
        if (2 * a <= n) st_c(acc_p + 2 * (2 * a), cadd(ld_c(acc_p + 2 * (2 * a)), tev));
      }
      if (loop) {
        const int i = lane >> 1, half = lane & 1;
        cplx acc = mkc(0.0, 0.0);
        if (i < rows)
          for (int t = half; t < s; t += 2) acc = cfma(ld_c(Pb + (i * ps + t) * 2), ld_c(Dv + t * 2), acc);
        acc.re += shfl_xor_d(acc.re, 1);
        acc.im += shfl_xor_d(acc.im, 1);
        if (half == 0 && i < 16) st_c(Y + (i * (h + 1) + a) * 2, i < rows ? acc : mkc(0.0, 0.0));
      }
      __syncwarp();
      double* tmp = Pa; Pa = Pb; Pb = tmp;
    }
    if (loop) {
      // v_k += 1/2 sum_i y_a[i^1] y_b[i],  a = (k-1)/2, b = k-1-a
      for (int k = 1; k <= n; ++k) {
        const int aa = (k - 1) >> 1, bb = k - 1 - aa;
        cplx t = mkc(0.0, 0.0);
        if (lane < rows) t = cmul(ld_c(Y + ((lane ^ 1) * (h + 1) + aa) * 2), ld_c(Y + (lane * (h + 1) + bb) * 2));
        t = warp_sum_c(t);
        if (lane == 0) st_c(acc_v + 2 * k, cadd(ld_c(acc_v + 2 * k), cscale(t, 0.5)));
      }
    }
    __syncwarp();
  }

  // ---- Newton recurrence, every lane redundantly (identical values)
  if (lane == 0) {
    for (int k = 1; k <= n; ++k) {
      cplx g = cscale(ld_c(acc_p + 2 * k), 0.5);
      if (loop) g = cadd(g, cscale(ld_c(acc_v + 2 * k), (double)k));
      st_c(kg + 2 * k, g);
    }
    st_c(ev, mkc(1.0, 0.0));
    for (int j = 1; j <= n; ++j) {
      cplx acc = mkc(0.0, 0.0);
      for (int k = 1; k <= j; ++k) acc = cadd(acc, cmul(ld_c(kg + 2 * k), ld_c(ev + 2 * (j - k))));
      st_c(ev + 2 * j, mkc(acc.re / j, acc.im / j));
    }
  }
  __syncwarp();
  cplx coeff = ld_c(ev + 2 * n);
  __syncwarp();
  return ((n - m) & 1) ? cneg(coeff) : coeff;
}

}  // namespace gbsb
