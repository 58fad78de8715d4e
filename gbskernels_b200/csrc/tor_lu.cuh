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

#include "cert.cuh"
#include "gbs_common.cuh"

namespace gbsb {

constexpr int kTorLuMaxModes = 12;               // dim 24, the reference's GPU cap
constexpr int kTorLuMaxDim = 2 * kTorLuMaxModes;  // 24
constexpr int kTorLuStride = kTorLuMaxDim + 1;    // complex row stride (bank spread)

// workspace: the minor (complex, stride kTorLuStride), 64 doubles of index space,
// and for the certified tier one radius per entry of the minor
__host__ __device__ inline int tor_lu_ws_doubles(bool cert = false) {
  return 2 * kTorLuMaxDim * kTorLuStride + 64 + (cert ? kTorLuMaxDim * kTorLuStride : 0);
}

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

// ---- certified helpers: the midpoints are the binary64 operations above, the
// radii are bounded a posteriori (no error model of Smith's division or of the
// square root is assumed).
__device__ __forceinline__ double rd_abs_c(cplx z) {
  return rd_sqrt(rd_add(rd_mul(z.re, z.re), rd_mul(z.im, z.im)));
}

// |a / b - tor_cdiv(a, b)| for exact a, b: |a - q b| / |b| with the residual
// a - fl(q b) carried as a ball (complex product 4u|q||b|, subtraction u|.|).
__device__ __forceinline__ double tor_cdiv_err(cplx a, cplx b, cplx q, double blo) {
  const cplx qb = cmul(q, b);
  const cplx res = csub(a, qb);
  double r = ru_add(ru_abs_c(res), ru_mul(4.0 * kU, ru_mul(ru_abs_c(q), ru_abs_c(b))));
  r = ru_add(r, ru_add(ru_mul(kUc, ru_abs_c(res)), 4.0 * kUfl));
  return ru_div(r, blo);
}

// Ball quotient (a +- ra) / (b +- rb) with midpoint tor_cdiv(a, b):
// |a*/b* - q| <= |a/b - q| + (ra + |a/b| rb) / (|b| - rb).  Infinite radius when
// the divisor's ball reaches zero.
__device__ __forceinline__ cball tor_cdiv_ball(cball a, cball b) {
  cball o;
  o.z = tor_cdiv(a.z, b.z);
  const double blo = rd_abs_c(b.z);
  if (!(blo > b.r)) {
    o.r = INFINITY;
    return o;
  }
  const double e0 = tor_cdiv_err(a.z, b.z, o.z, blo);
  const double qa = ru_add(ru_abs_c(o.z), e0);  // >= |a / b|
  o.r = ru_add(e0, ru_div(ru_add(a.r, ru_mul(qa, b.r)), rd_sub(blo, b.r)));
  return o;
}

// Ball of 1 / sqrt(z*), |z* - z| <= ez, principal branch, midpoint
// tor_cdiv(1, tor_csqrt_principal(z)).  Refused (infinite radius) when the ball
// reaches the branch cut (-inf, 0] or is not small against |z|.  With s the
// computed root and delta >= |s^2 - z|: s and sqrt(z) lie in the same quadrant
// (the root takes the sign of Im z), so |s + sqrt(z)| >= |s| and
// |s - sqrt(z)| <= delta / |s|; sqrt(z) and sqrt(z*) differ in argument by at most
// asin(ez/|z|) / 2 < 90 degrees, so |sqrt(z) - sqrt(z*)| <= ez / sqrt|z|; then
// |1/sqrt(z*) - 1/s| <= e_s / (|s| (|s| - e_s)) and the division by s adds its
// own a-posteriori error.
__device__ __forceinline__ cball tor_inv_sqrt_ball(cball z) {
  cball o;
  const cplx s = tor_csqrt_principal(z.z);
  o.z = tor_cdiv(mkc(1.0, 0.0), s);
  const double zlo = rd_abs_c(z.z);
  const bool near_cut = (z.z.re <= 0.0 && fabs(z.z.im) <= z.r);
  if (!(zlo > 0.0) || !(z.r <= 0.5 * zlo) || near_cut || !isfinite(z.r)) {
    o.r = INFINITY;
    return o;
  }
  const cplx s2 = cmul(s, s);
  const cplx d = csub(s2, z.z);
  const double sa = ru_abs_c(s);
  double delta = ru_add(ru_abs_c(d), ru_mul(4.0 * kU, ru_mul(sa, sa)));
  delta = ru_add(delta, ru_add(ru_mul(kUc, ru_abs_c(d)), 4.0 * kUfl));
  const double slo = rd_abs_c(s);
  if (!(slo > 0.0)) {
    o.r = INFINITY;
    return o;
  }
  const double es = ru_add(ru_div(delta, slo), ru_div(z.r, rd_sqrt(zlo)));
  if (!(es < slo)) {
    o.r = INFINITY;
    return o;
  }
  const double e1 = ru_div(es, rd_mul(slo, rd_sub(slo, es)));
  o.r = ru_add(e1, tor_cdiv_err(mkc(1.0, 0.0), s, o.z, slo));
  return o;
}

// Signed term of subset `mask` of the complex 2n x 2n O (interleaved).  Every lane
// returns the same value.  ws: this warp's workspace (tor_lu_ws_doubles(CERT)).
// CERT: a radius rides along with every entry of the minor (the ball arithmetic of
// cert.cuh; the division and the root bounded a posteriori); the midpoints are the
// binary64 tier's operations, so the value is the fp64 value bit for bit.
template <bool CERT>
static __device__ cball tor_lu_term(const double* __restrict__ Oc, int n, uint32_t mask, double* ws, int lane,
                                    bool& singular) {
  const int m = __popc(mask);
  const int dim = 2 * n;
  if (m == 0) return cball{((n & 1) ? mkc(-1.0, 0.0) : mkc(1.0, 0.0)), 0.0};
  const int mm = 2 * m;
  int* idx = reinterpret_cast<int*>(ws + 2 * kTorLuMaxDim * kTorLuStride);
  double* R = ws + 2 * kTorLuMaxDim * kTorLuStride + 64;  // radii (certified tier)
  if (lane < mm) {
    // lane -> component: the lane-th set mode (x part) or, past m, its p part
    const int t = lane < m ? lane : lane - m;
    uint32_t mk = mask;
    for (int u = 0; u < t; ++u) mk &= mk - 1;
    const int mode = __ffs(mk) - 1;
    idx[lane] = lane < m ? mode : mode + n;
  }
  __syncwarp();
  // I - O_S, row r owned by lane r (off the diagonal the negation is exact; the
  // diagonal 1 - o rounds once)
  double* M = ws;
  if (lane < mm) {
    const int gr = idx[lane];
    for (int c = 0; c < mm; ++c) {
      const int gc = idx[c];
      const double* o = Oc + 2 * ((size_t)gr * dim + gc);
      const cplx v = mkc((gr == gc ? 1.0 : 0.0) - o[0], -o[1]);
      st_c(M + 2 * (lane * kTorLuStride + c), v);
      if constexpr (CERT) R[lane * kTorLuStride + c] = gr == gc ? ru_add(ru_mul(kUc, fabs(v.re)), kUfl) : 0.0;
    }
  }
  __syncwarp();
  bool used = lane >= mm;  // rows already chosen as pivots (idle lanes count as used)
  cball det{mkc(1.0, 0.0), 0.0};
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
      return cball{mkc(0.0, 0.0), CERT ? INFINITY : 0.0};
    }
    // the permutation's parity: rows before `who` not used yet are passed over
    const unsigned free_below = __ballot_sync(0xffffffffu, !used && lane < who);
    inversions += __popc(free_below);
    const cball piv{ld_c(M + 2 * (who * kTorLuStride + c)), CERT ? R[who * kTorLuStride + c] : 0.0};
    if constexpr (CERT) det = cb_mul(det, piv);
    else det.z = cmul(det.z, piv.z);
    if (lane == who) used = true;
    if (!used) {
      cball f;
      if constexpr (CERT) {
        f = tor_cdiv_ball(cball{ld_c(M + 2 * (lane * kTorLuStride + c)), R[lane * kTorLuStride + c]}, piv);
      } else {
        f.z = tor_cdiv(ld_c(M + 2 * (lane * kTorLuStride + c)), piv.z);
      }
      for (int j = c + 1; j < mm; ++j) {
        const cplx pj = ld_c(M + 2 * (who * kTorLuStride + j));
        const cplx mj = ld_c(M + 2 * (lane * kTorLuStride + j));
        if constexpr (CERT) {
          const cball prod = cb_mul(f, cball{pj, R[who * kTorLuStride + j]});
          const cball nm = cb_add(cball{mj, R[lane * kTorLuStride + j]}, cb_neg(prod));
          st_c(M + 2 * (lane * kTorLuStride + j), nm.z);
          R[lane * kTorLuStride + j] = nm.r;
        } else {
          st_c(M + 2 * (lane * kTorLuStride + j), csub(mj, cmul(f.z, pj)));
        }
      }
    }
    __syncwarp();
  }
  if (inversions & 1) det.z = cneg(det.z);
  cball t;
  if constexpr (CERT) {
    t = tor_inv_sqrt_ball(det);
  } else {
    t.z = tor_cdiv(mkc(1.0, 0.0), tor_csqrt_principal(det.z));
    t.r = 0.0;
  }
  if ((n - m) & 1) t.z = cneg(t.z);
  return t;
}

}  // namespace gbsb
