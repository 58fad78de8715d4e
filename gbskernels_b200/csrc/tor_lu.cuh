// tor_lu.cuh -- torontonian of a COMPLEX O by subset LU determinants (binary64).
//
// tor(O) = sum_{S subset [n]} (-1)^(n-|S|) / sqrt(det(I - O_S)),  xxpp ordering,
// with the principal complex square root.  Reference: core/torontonian.cu:29-110
// (det_lu with partial pivoting, csqrt_principal, tor_subset_term) and
// cpu_ref/torontonian.py:48-64.  A complex O has no Cholesky factor, so the
// reference (and this path) factors every minor independently; the real physical
// domain goes through the prefix-Cholesky walk of tor_warp.cuh instead.
//
// B200 mapping: one warp per subset at a time.  The minor (m = 2|S| <= 24 rows,
// complex) is staged in the warp's shared workspace, lane r owns row r; each
// elimination step picks the pivot row by a warp arg-max of |M[r][c]|^2 over the
// rows not yet used (no row is moved: the pivot order is tracked), and every other
// active row subtracts f * (pivot row) with the pivot row read as a shared-memory
// broadcast.  det = sign * prod of pivots; the sign of the permutation follows
// from the pivot order.  Items are ranges of subset masks.
#pragma once

#include "gbs_common.cuh"

namespace gbsb {

constexpr int kTorLuMaxModes = 12;               // dim 24, the reference's GPU cap
constexpr int kTorLuMaxDim = 2 * kTorLuMaxModes;  // 24
constexpr int kTorLuStride = kTorLuMaxDim + 1;    // complex row stride (bank spread)

__host__ __device__ inline int tor_lu_ws_doubles() { return 2 * kTorLuMaxDim * kTorLuStride + 64; }

// a / b by Smith's method (R. L. Smith, CACM 5(8), 1962): scale by the larger
// component of b so the intermediate products cannot overflow.
__device__ __forceinline__ cplx tor_cdiv(cplx a, cplx b) {
  if (fabs(b.re) >= fabs(b.im)) {
    const double r = b.im / b.re, den = b.re + b.im * r;
    return mkc((a.re + a.im * r) / den, (a.im - a.re * r) / den);
  }
  const double r = b.re / b.im, den = b.im + b.re * r;
  return mkc((a.re * r + a.im) / den, (a.im * r - a.re) / den);
}

__device__ __forceinline__ cplx tor_csqrt_principal(cplx z) {
  const double r = hypot(z.re, z.im);
  double re = sqrt(0.5 * (r + z.re));
  double im = sqrt(0.5 * (r - z.re));
  if (z.im < 0.0) im = -im;
  return mkc(re, im);
}

// Signed term of subset `mask` of the complex 2n x 2n O (interleaved).  Every lane
// returns the same value.  ws: this warp's workspace (tor_lu_ws_doubles()).
static __device__ cplx tor_lu_term(const double* __restrict__ Oc, int n, uint32_t mask, double* ws, int lane,
                            bool& singular) {
  const int m = __popc(mask);
  const int dim = 2 * n;
  if (m == 0) return ((n & 1) ? mkc(-1.0, 0.0) : mkc(1.0, 0.0));
  const int mm = 2 * m;
  int* idx = reinterpret_cast<int*>(ws + 2 * kTorLuMaxDim * kTorLuStride);
  if (lane < mm) {
    // lane -> component: the lane-th set mode (x part) or, past m, its p part
    const int t = lane < m ? lane : lane - m;
    uint32_t mk = mask;
    for (int u = 0; u < t; ++u) mk &= mk - 1;
    const int mode = __ffs(mk) - 1;
    idx[lane] = lane < m ? mode : mode + n;
  }
  __syncwarp();
  // I - O_S, row r owned by lane r
  double* M = ws;
  if (lane < mm) {
    const int gr = idx[lane];
    for (int c = 0; c < mm; ++c) {
      const int gc = idx[c];
      const double* o = Oc + 2 * ((size_t)gr * dim + gc);
      st_c(M + 2 * (lane * kTorLuStride + c), mkc((gr == gc ? 1.0 : 0.0) - o[0], -o[1]));
    }
  }
  __syncwarp();
  bool used = lane >= mm;  // rows already chosen as pivots (idle lanes count as used)
  cplx det = mkc(1.0, 0.0);
  int inversions = 0;      // parity of the pivot order as a permutation
  for (int c = 0; c < mm; ++c) {
    // arg-max of |M[r][c]|^2 over unused rows (ties: the lowest row)
    double best = -1.0;
    if (!used) {
      const cplx v = ld_c(M + 2 * (lane * kTorLuStride + c));
      best = v.re * v.re + v.im * v.im;
    }
    int who = lane;
#pragma unroll
    for (int s = 16; s > 0; s >>= 1) {
      const double ob = shfl_xor_d(best, s);
      const int ow = __shfl_xor_sync(0xffffffffu, who, s);
      if (ob > best || (ob == best && ow < who)) {
        best = ob;
        who = ow;
      }
    }
    if (!(best > 0.0)) {
      singular = true;
      return mkc(0.0, 0.0);
    }
    // the permutation's parity: rows before `who` not used yet are passed over
    const unsigned free_below = __ballot_sync(0xffffffffu, !used && lane < who);
    inversions += __popc(free_below);
    const cplx piv = ld_c(M + 2 * (who * kTorLuStride + c));
    det = cmul(det, piv);
    if (lane == who) used = true;
    if (!used) {
      const cplx f = tor_cdiv(ld_c(M + 2 * (lane * kTorLuStride + c)), piv);
      for (int j = c + 1; j < mm; ++j) {
        const cplx pj = ld_c(M + 2 * (who * kTorLuStride + j));
        const cplx mj = ld_c(M + 2 * (lane * kTorLuStride + j));
        st_c(M + 2 * (lane * kTorLuStride + j), csub(mj, cmul(f, pj)));
      }
    }
    __syncwarp();
  }
  if (inversions & 1) det = cneg(det);
  const cplx t = tor_cdiv(mkc(1.0, 0.0), tor_csqrt_principal(det));
  return ((n - m) & 1) ? cneg(t) : t;
}

}  // namespace gbsb
