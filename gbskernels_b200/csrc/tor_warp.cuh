// tor_warp.cuh -- torontonian by a warp-cooperative prefix-Cholesky walk with a
// 32-subset register tail per prefix leaf (binary64, kappa and certified tiers).
//
// tor(O) = sum_{S subset [k]} (-1)^(k-|S|) / sqrt(det((I - O)_S)),  xxpp ordering,
// where including mode j puts rows / columns j and j + k of M = I - O in the minor.
// Reference algorithm: the recursive prefix Cholesky of core/tor_recursive.cu:41-115
// (cpu_ref/tor_recursive.py:46-100): the subsets are walked in binary-counter order,
// including a mode appends its two rows to one Cholesky factor, det = prod of the
// squared pivots.
//
// B200 mapping (this repository's design):
//   * the last r = min(k, 5) modes form the TAIL, the first q = k - r the PREFIX.
//     The tail rows sit at the bottom of every column of the factor: for a prefix
//     subset S with factor L of M_S, column u holds L[t][u] (prefix rows t > u)
//     followed by W[u][.] = (L^{-1} M_{S,T})[u][.], and the Schur complement
//     Z = M_TT - W^T W is kept per depth (Zd[c] after c prefix modes), updated by
//     the two new W rows of each append;
//   * one warp walks the prefix subsets of a work item (a fixed pattern over the
//     first g prefix modes, then all subsets of the prefix modes [g, q)).  Appending
//     a mode computes its two factor rows and two W rows in one forward substitution:
//     lanes own residual slots x (prefix columns, the two new diagonal slots, the
//     2r tail columns), the owner of step v scales its residual by 1 / L[v][v] and
//     broadcasts it, every lane updates with column v (contiguous in shared memory);
//   * at every prefix leaf, lane l takes the tail subset T' = l: Z~ = Z with the
//     rows / columns of the excluded tail modes replaced by the identity (the same
//     determinant, and the same rounded operations as factoring the compressed
//     matrix, since the extra terms are exact zeros), factored in registers, and the
//     32 signed terms are summed by a fixed butterfly;
//   * the factor, Zd and the pivot reciprocals live in the warp's shared workspace
//     (about 18 KB at 24 modes): no local memory.
//
// Pivots: the factor keeps 1 / L[j][j] = rsqrt(s_j) (s_j the pivot before the root);
// off-diagonal entries are s_ij * rsqrt(s_j), det = prod s_j, term = rsqrt(det).
// CUDA documents double rsqrt to 1 ulp; the certified bound below assumes 2 ulp
// (relative error <= 4u), so it does not lean on the last ulp of that figure.
//
// Certified tier: the binary64 walk is the fp64 tier's (bit-identical value) and each
// term gets an a-posteriori radius.  Define L^_jj := 1 / rsqrt(s_j) (exact real).  For
// a subset of dimension m the computed factor then satisfies L^L^T = A + F with
// |F_ij| <= c_m D_i D_j (Cholesky backward error: each entry is an inner product of
// <= m fused terms and one scaling, the diagonal carries (1 + 4u)^2 from rsqrt, so
// gamma_{m+10} covers it; D_i = fl(sqrt(fl(1 - O_ii)))), hence det(L^)^2 =
// det(A) det(I + X) with ||X|| <= eta_m = m c_m / sigma, sigma a rigorous lower bound
// of lambda_min(D^-1 M D^-1) -- valid for every principal submatrix by Cauchy
// interlacing, so ONE bound per instance certifies all 2^k subsets.  sigma is proved
// per instance by a binary64 Cholesky of D^-1 M D^-1 - sigma I that succeeds (success
// implies lambda_min >= -g tr / (1 - g), g = gamma_{2k+10}; Weyl for the rounding of
// the scaled matrix), at a sigma guessed by inverse iteration.  The term radius is
// |t^| rho_m with rho_m from eta_m, the pivot product (m + 1 roundings), the rsqrt
// of every pivot and the final rsqrt (tor_cert_rho).
#pragma once

#include <type_traits>

#include "cert.cuh"
#include "gbs_common.cuh"

namespace gbsb {

constexpr int kTorTail = 5;                        // tail modes (2^5 subsets = 32 lanes)
constexpr int kTorTD = 2 * kTorTail;               // tail rows (10)
constexpr int kTorZE = kTorTD * (kTorTD + 1) / 2;  // packed lower tail entries (55)

struct TorWLayout {
  int col_off, inv_off, zd_off, det_off, gidx_off, id_off, rho_off, total;  // in doubles
};

// rows = 2q prefix rows; column u holds rows - u prefix slots + 10 tail slots.
__host__ __device__ inline int tor_col_base(int u, int rows) { return u * (rows + kTorTD) - (u * (u - 1)) / 2; }

__host__ __device__ inline TorWLayout tor_w_layout(int kmax, bool cert) {
  TorWLayout Lw;
  const int q = kmax > kTorTail ? kmax - kTorTail : 0;
  const int rows = 2 * q;
  Lw.col_off = 0;
  Lw.inv_off = Lw.col_off + tor_col_base(rows, rows) + 1;
  Lw.zd_off = Lw.inv_off + rows + 1;
  Lw.det_off = Lw.zd_off + (q + 1) * kTorZE;
  Lw.gidx_off = Lw.det_off + q + 2;
  Lw.id_off = Lw.gidx_off + (rows + 2) / 2;  // packed 10 x 10 identity (excluded tail rows)
  Lw.rho_off = Lw.id_off + kTorZE + 1;
  int total = Lw.rho_off + (cert ? 2 * kmax + 2 : 0);
  if (cert) {  // the sigma proof factors a packed 2k x 2k matrix (+ 2k scalings) in the col / zd region
    const int need = (2 * kmax) * (2 * kmax + 1) / 2 + 2 * kmax + 8;
    if (Lw.det_off < need) {
      const int shift = need - Lw.det_off;
      Lw.det_off += shift;
      Lw.gidx_off += shift;
      Lw.id_off += shift;
      Lw.rho_off += shift;
      total += shift;
    }
  }
  Lw.total = (total + 3) & ~3;
  return Lw;
}

__device__ __forceinline__ double tor_m(const double* __restrict__ Oc, int dim, int a, int b) {
  // entry of M = I - O from the complex-interleaved input (real part)
  const double o = Oc[2 * (a * dim + b)];
  return a == b ? 1.0 - o : -o;
}

// global component index of tail row jt (x of mode q + jt/2, or its p)
__device__ __forceinline__ int tor_tail_g(int jt, int q, int k) { return (jt & 1) ? q + (jt >> 1) + k : q + (jt >> 1); }

// packed lower index e -> (row i, column jj), i >= jj, i < 10
__device__ __forceinline__ void tor_tri_ij(int e, int& i, int& jj) {
  i = 0;
  while ((i + 1) * (i + 2) / 2 <= e) ++i;
  jj = e - i * (i + 1) / 2;
}

// Append prefix mode j (global components j and j + k) as rows R0 = 2c, R1 = 2c + 1.
// Writes the two factor rows into columns 0..R0 (and L[R1][R0]), the two W rows
// into the tail slots of columns R0 and R1, inv[R0], inv[R1], detat[c + 1] and
// Zd[c + 1].  Returns false when a pivot is not positive (the walk continues with a
// unit pivot; the instance is flagged).  (zi, zj): this lane's Zd entries.
__device__ __forceinline__ bool tor_w_append(const double* __restrict__ Oc, int k, int q, int r, int j, int c,
                                             double* col, double* inv, double* zd, double* detat, int* gidx,
                                             int lane, const int (&zi)[2], const int (&zj)[2]) {
  const int dim = 2 * k;
  const int rows = 2 * q;
  const int R0 = 2 * c, R1 = R0 + 1;
  const int gR0 = j, gR1 = j + k;
  const int nx = R0 + 2 * r;
  if (lane == 0) {
    gidx[R0] = gR0;
    gidx[R1] = gR1;
  }
  // residual slots x = lane, lane + 32: x < R0 = prefix column x (reads L[x][v], at
  // column offset x - v, while v < x), R0 <= x < R0 + 2r = tail column x - R0
  // (reads W[v][x - R0] at offset rows + x - R0 - v), beyond = idle
  double a[2], b[2];
  int lim[2], off[2];  // a slot reads column v at offset off - v while v < lim
#pragma unroll
  for (int h = 0; h < 2; ++h) {
    const int x = lane + 32 * h;
    a[h] = 0.0;
    b[h] = 0.0;
    lim[h] = x < R0 ? x : (x < nx ? R0 : 0);
    off[h] = x < R0 ? x : rows + (x - R0);
    if (x < R0) {
      const int gc = gidx[x];
      a[h] = tor_m(Oc, dim, gR0, gc);
      b[h] = tor_m(Oc, dim, gR1, gc);
    } else if (x < nx) {
      const int gT = tor_tail_g(x - R0, q, k);
      a[h] = tor_m(Oc, dim, gR0, gT);
      b[h] = tor_m(Oc, dim, gR1, gT);
    }
  }
  // the new 2 x 2 diagonal block, accumulated in every lane from the broadcast values
  double d00 = tor_m(Oc, dim, gR0, gR0), d10 = tor_m(Oc, dim, gR1, gR0), d11 = tor_m(Oc, dim, gR1, gR1);
  // forward substitution over the existing columns v < R0 (owners of v < 32 hold the
  // residual in slot 0, the others in slot 1)
  double* cv = col;  // column v starts at tor_col_base(v, rows)
  // NS residual slots per lane take part: when every slot fits one warp (nx <= 32,
  // warp-uniform) the second slot is idle throughout and its update is skipped
  // (it would be fma(-0, l, 0) == 0: the values do not change)
  auto step = [&](auto ns, int v, double av, double bv) {
    constexpr int NS = decltype(ns)::value;
    const double iv = inv[v];
    const double l0 = av * iv, l1 = bv * iv;
    if (lane == (v & 31)) {
      cv[R0 - v] = l0;
      cv[R1 - v] = l1;
    }
#pragma unroll
    for (int h = 0; h < NS; ++h) {
      double e = 0.0;  // 0 for finished or idle slots: fma(-0, l, a) == a
      if (v < lim[h]) e = cv[off[h] - v];
      a[h] = fma(-e, l0, a[h]);
      b[h] = fma(-e, l1, b[h]);
    }
    d00 = fma(-l0, l0, d00);
    d10 = fma(-l0, l1, d10);
    d11 = fma(-l1, l1, d11);
    cv += rows + kTorTD - v;
  };
  const int v1 = R0 < 32 ? R0 : 32;
  if (nx <= 32) {
    for (int v = 0; v < v1; ++v)
      step(std::integral_constant<int, 1>{}, v, __shfl_sync(0xffffffffu, a[0], v), __shfl_sync(0xffffffffu, b[0], v));
  } else {
    for (int v = 0; v < v1; ++v)
      step(std::integral_constant<int, 2>{}, v, __shfl_sync(0xffffffffu, a[0], v), __shfl_sync(0xffffffffu, b[0], v));
    for (int v = 32; v < R0; ++v)
      step(std::integral_constant<int, 2>{}, v, __shfl_sync(0xffffffffu, a[1], v & 31),
           __shfl_sync(0xffffffffu, b[1], v & 31));
  }
  // the two pivots (identical in every lane)
  double s0 = d00;
  bool ok = s0 > 0.0;
  if (!ok) s0 = 1.0;
  const double i0 = rsqrt(s0);
  const double l10 = d10 * i0;
  double s1 = fma(-l10, l10, d11);
  if (!(s1 > 0.0)) {
    ok = false;
    s1 = 1.0;
  }
  const double i1 = rsqrt(s1);
  double* c0 = col + tor_col_base(R0, rows);
  double* c1 = col + tor_col_base(R1, rows);
#pragma unroll
  for (int h = 0; h < 2; ++h) {
    const int x = lane + 32 * h;
    if (x >= R0 && x < nx) {
      const int jt = x - R0;
      const double w0 = a[h] * i0;
      const double w1 = fma(-w0, l10, b[h]) * i1;
      c0[rows - R0 + jt] = w0;
      c1[rows - R1 + jt] = w1;
    }
  }
  if (lane == 0) {
    c0[1] = l10;
    inv[R0] = i0;
    inv[R1] = i1;
    detat[c + 1] = detat[c] * s0 * s1;
  }
  __syncwarp();
  // Zd[c + 1] = Zd[c] - w0 w0^T - w1 w1^T  (packed lower, tail rows < 2r)
  const double* zs = zd + c * kTorZE;
  double* zt = zd + (c + 1) * kTorZE;
  const double* w0p = c0 + rows - R0;
  const double* w1p = c1 + rows - R1;
#pragma unroll
  for (int h = 0; h < 2; ++h) {
    const int e = lane + 32 * h;
    if (e < kTorZE) {
      double z = zs[e];
      if (zi[h] < 2 * r) {
        z = fma(-w0p[zi[h]], w0p[zj[h]], z);
        z = fma(-w1p[zi[h]], w1p[zj[h]], z);
      }
      zt[e] = z;
    }
  }
  __syncwarp();
  return ok;
}

// One prefix leaf: every lane l < 2^r factors Z~ for the tail subset l.  Returns the
// lane's signed term (0 for idle lanes); ok is cleared on a non-positive pivot and
// the term dimension m = 2 (c + |T'|) is returned for the certified radius.
// Rows of excluded tail modes are read from the packed identity zid, and their
// pivot reciprocal is set to 0: every entry in an excluded row or column is then an
// exact zero and every fused term it feeds is exact, so the included entries see
// the same rounded operations as the factorisation of the compressed matrix.
__device__ __forceinline__ double tor_w_leaf(const double* zc, const double* zid, int r, int c, int k, double detc,
                                             int lane, bool& ok, int& m) {
  double term = 0.0;
  m = 0;
  if (lane < (1 << r)) {
    const int td = 2 * r;
    double Lz[kTorZE];  // off-diagonal entries (the diagonal slots stay unused)
    double iv[kTorTD];  // 1 / L[i][i] (0 for excluded rows)
    double det = 1.0;
#pragma unroll
    for (int i = 0; i < kTorTD; ++i) {
      const bool in_i = i < td && ((lane >> (i >> 1)) & 1);
      const double* zr = (in_i ? zc : zid) + i * (i + 1) / 2;
#pragma unroll
      for (int jj = 0; jj <= i; ++jj) {
        const int e = i * (i + 1) / 2 + jj;
        double s = zr[jj];
#pragma unroll
        for (int u = 0; u < jj; ++u) s = fma(-Lz[i * (i + 1) / 2 + u], Lz[jj * (jj + 1) / 2 + u], s);
        if (jj < i) {
          Lz[e] = s * iv[jj];
        } else {
          if (!(s > 0.0)) {
            ok = false;
            s = 1.0;
          }
          iv[i] = in_i ? rsqrt(s) : 0.0;  // excluded rows: s == 1 exactly
          det *= s;
        }
      }
    }
    const int nin = __popc(lane);
    m = 2 * (c + nin);
    const double t = rsqrt(detc * det);
    term = ((k - c - nin) & 1) ? -t : t;
  }
  return term;
}

// ------------------------------------------------------------ certified prologue
// Rigorous lower bound sigma of lambda_min(D^-1 M D^-1), D_i = fl(sqrt(fl(1 - O_ii))),
// for the whole 2k x 2k matrix; <= 0 when none could be proved.  Also returns a lower
// bound of min D_i^2 for the underflow term.  Scratch (warp-private shared memory):
// the packed lower (2k)(2k+1)/2 matrix at S, then 2k scalings.
//   H^_ij = fl(fl(m_ij * fl(1/D_i)) * fl(1/D_j)) is within gamma_5 |h_ij| of the exact
//   scaled entry, so ||H^ - H||_2 <= ||H^ - H||_F <= gamma_5 / (1 - gamma_5) ||H^||_F.
//   A binary64 Cholesky of B = fl(H^ - s I) that completes proves lambda_min(B) >=
//   -g tr(B) / (1 - g), g = gamma_{2k+10} (backward error of the factorisation, the
//   rsqrt pivots included); with the rounding of the diagonal shift (u sum |b_ii|),
//   lambda_min(H) >= s - g tr / (1 - g) - ||E||.
//   The trial shift comes from inverse iteration with the factor of H^ itself.
static __device__ __noinline__ double tor_cert_sigma(const double* __restrict__ Oc, int k, double* S, int lane, double& dmin2) {
  const int dim = 2 * k;
  const int np = dim * (dim + 1) / 2;
  double* dinv = S + np;
  double dm = 1e300;
  bool okd = true;
  for (int i = lane; i < dim; i += 32) {
    const double mii = 1.0 - Oc[2 * (i * dim + i)];
    if (!(mii > 0.0)) okd = false;
    const double di = mii > 0.0 ? sqrt(mii) : 1.0;
    dinv[i] = 1.0 / di;
    dm = fmin(dm, __dmul_rd(di, di));
  }
  okd = __all_sync(0xffffffffu, okd);
#pragma unroll
  for (int mm = 16; mm > 0; mm >>= 1) dm = fmin(dm, shfl_xor_d(dm, mm));
  dmin2 = dm;
  __syncwarp();
  if (!okd) return -1.0;
  auto unpack = [&](int e, int& i, int& jj) {
    i = (int)((sqrt(8.0 * e + 1.0) - 1.0) * 0.5);
    while (i * (i + 1) / 2 > e) --i;
    while ((i + 1) * (i + 2) / 2 <= e) ++i;
    jj = e - i * (i + 1) / 2;
  };
  auto hval = [&](int i, int jj) { return (tor_m(Oc, dim, i, jj) * dinv[i]) * dinv[jj]; };
  double fro2 = 0.0;
  for (int e = lane; e < np; e += 32) {
    int i, jj;
    unpack(e, i, jj);
    const double h = hval(i, jj);
    fro2 = ru_fma(h, h, fro2);
    if (i != jj) fro2 = ru_fma(h, h, fro2);
  }
  fro2 = warp_sum_ru(fro2);
  const double g5 = gamma_ru(5.0, kU);
  const double eh = ru_mul(ru_div(g5, rd_sub(1.0, g5)), ru_sqrt(fro2));
  const double gm = gamma_ru((double)(dim + 10), kU);
  // factor B = fl(H^ - sig I) in place (right-looking, packed lower; the diagonal
  // slot of column j ends holding rsqrt of its pivot); on success return the proved
  // bound sig - tau - ||E||, else -1
  auto attempt = [&](double sig) -> double {
    double trace = 0.0;
    for (int e = lane; e < np; e += 32) {
      int i, jj;
      unpack(e, i, jj);
      double h = hval(i, jj);
      if (i == jj) {
        h = h - sig;
        trace = ru_add(trace, fabs(h));
      }
      S[e] = h;
    }
    trace = warp_sum_ru(trace);
    __syncwarp();
    for (int jc = 0; jc < dim; ++jc) {
      const double p = S[jc * (jc + 1) / 2 + jc];
      if (!(p > 0.0)) {  // warp-uniform (every lane read the same word)
        __syncwarp();
        return -1.0;
      }
      const double id = rsqrt(p);
      __syncwarp();
      if (lane == 0) S[jc * (jc + 1) / 2 + jc] = id;
      for (int i = jc + 1 + lane; i < dim; i += 32) S[i * (i + 1) / 2 + jc] *= id;
      __syncwarp();
      for (int i = jc + 1; i < dim; ++i) {
        const double lij = S[i * (i + 1) / 2 + jc];
        for (int l = jc + 1 + lane; l <= i; l += 32)
          S[i * (i + 1) / 2 + l] = fma(-lij, S[l * (l + 1) / 2 + jc], S[i * (i + 1) / 2 + l]);
      }
      __syncwarp();
    }
    const double tau = ru_div(ru_mul(gm, trace), rd_sub(1.0, gm));
    const double err = ru_add(eh, ru_mul(kUc, trace));
    return rd_sub(rd_sub(sig, tau), err);
  };
  if (attempt(0.0) < -0.5) return -1.0;  // H^ itself does not factor
  // inverse iteration x <- (L L^T)^{-1} x with the factor in S (slots x = lane, lane + 32)
  double x0 = lane < dim ? 1.0 + 0.01 * lane : 0.0;
  double x1 = lane + 32 < dim ? 1.0 + 0.01 * (lane + 32) : 0.0;
  double mu = 1.0;
  for (int it = 0; it < 5; ++it) {
    for (int j = 0; j < dim; ++j) {  // L y = x
      const double yj = __shfl_sync(0xffffffffu, (j >> 5) ? x1 : x0, j & 31) * S[j * (j + 1) / 2 + j];
      if (lane == (j & 31)) {
        if (j >> 5) x1 = yj;
        else x0 = yj;
      }
      if (lane > j && lane < dim) x0 = fma(-S[lane * (lane + 1) / 2 + j], yj, x0);
      if (lane + 32 > j && lane + 32 < dim) x1 = fma(-S[(lane + 32) * (lane + 33) / 2 + j], yj, x1);
    }
    for (int j = dim - 1; j >= 0; --j) {  // L^T z = y
      const double zj = __shfl_sync(0xffffffffu, (j >> 5) ? x1 : x0, j & 31) * S[j * (j + 1) / 2 + j];
      if (lane == (j & 31)) {
        if (j >> 5) x1 = zj;
        else x0 = zj;
      }
      const int r0 = j * (j + 1) / 2;
      if (lane < j) x0 = fma(-S[r0 + lane], zj, x0);
      if (lane + 32 < j) x1 = fma(-S[r0 + lane + 32], zj, x1);
    }
    double nn = x0 * x0 + x1 * x1;
#pragma unroll
    for (int mm = 16; mm > 0; mm >>= 1) nn += shfl_xor_d(nn, mm);
    mu = sqrt(nn);  // ~ 1 / lambda_min once converged (x had unit norm)
    if (!(mu > 0.0) || !isfinite(mu)) return -1.0;
    x0 /= mu;
    x1 /= mu;
  }
  const double est = 1.0 / mu;  // >= lambda_min(H^) up to rounding
  double best = -1.0;
  const double fr[6] = {0.9, 0.7, 0.45, 0.2, 0.05, 0.01};
  for (int t = 0; t < 6 && best <= 0.0; ++t) best = attempt(fr[t] * est);
  return best;
}

// rho_m for m = 0..2k (a-posteriori relative radius of one term of dimension m),
// written to rho[]; +inf where m * eta_m is not below 1/2.  e_r = 4u bounds the
// relative error of rsqrt (2 ulp).
//   c_m   = (g/(1-g) + u/(1-u)) / (1-u)^2 + (m+10) ufl / dmin2,  g = gamma_{m+10}
//   eta_m = m c_m / sigma,   gp = gamma_{m+1} (pivot product)
//   t / t^ = sqrt(det(I+X) (1+theta_p)) prod_j (1+d_j) / (1+d_f), |d| <= e_r, so
//   Up = sqrt((1+gp) / (1 - m eta)) / ((1 - m e_r)(1 - e_r))
//   Lo = sqrt((1-gp)(1 - m eta)) (1 - m e_r) / (1 + e_r)
//   and rho = max(Up - 1, 1 - Lo) bounds |t - t^| / |t^|.
static __device__ __noinline__ void tor_cert_rho(double sigma, double dmin2, int k, double* rho, int lane) {
  const double er = 4.0 * kU;
  for (int m = lane; m <= 2 * k; m += 32) {
    double out;
    if (m == 0) {
      out = 0.0;  // empty minor: t = 1 exactly
    } else if (!(sigma > 0.0) || !(dmin2 > 0.0)) {
      out = INFINITY;
    } else {
      const double md = (double)m;
      const double g = gamma_ru(md + 10.0, kU);
      double cm = ru_add(ru_div(g, rd_sub(1.0, g)), ru_div(kU, rd_sub(1.0, kU)));
      cm = ru_div(cm, __dmul_rd(rd_sub(1.0, kU), rd_sub(1.0, kU)));
      cm = ru_add(cm, ru_div(ru_mul(md + 10.0, kUfl), dmin2));
      const double eta = ru_div(ru_mul(md, cm), sigma);
      const double meta = ru_mul(md, eta);
      const double mer = ru_mul(md, er);
      if (!(meta < 0.5) || !(mer < 0.5)) {
        out = INFINITY;
      } else {
        const double gp = gamma_ru(md + 1.0, kU);
        const double one_meta = rd_sub(1.0, meta);
        const double one_mer = rd_sub(1.0, mer);
        double up = ru_sqrt(ru_div(ru_add(1.0, gp), one_meta));
        up = ru_div(up, __dmul_rd(one_mer, rd_sub(1.0, er)));
        double lo = rd_sqrt(__dmul_rd(rd_sub(1.0, gp), one_meta));
        lo = __ddiv_rd(__dmul_rd(lo, one_mer), ru_add(1.0, er));
        out = fmax(ru_add(up, -1.0), ru_add(1.0, -lo));
      }
    }
    rho[m] = out;
  }
  __syncwarp();
}

// ------------------------------------------------------------ one work item
// Prefix pattern `pat` over the first g prefix modes, then every subset of the
// prefix modes [g, q) with its 2^r tail subsets.  KAPPA adds sum |term|, CERT the
// ball radius (aux).  Returns false when a pivot was not positive.
template <bool KAPPA, bool CERT>
static __device__ bool tor_warp_item(const double* __restrict__ Oc, int k, int g, uint32_t pat, double* ws,
                              const TorWLayout& Lw, const double* rho, int lane, double& total, double& aux) {
  const int dim = 2 * k;
  const int r = k < kTorTail ? k : kTorTail;
  const int q = k - r;
  double* col = ws + Lw.col_off;
  double* inv = ws + Lw.inv_off;
  double* zd = ws + Lw.zd_off;
  double* detat = ws + Lw.det_off;
  int* gidx = reinterpret_cast<int*>(ws + Lw.gidx_off);
  double* zid = ws + Lw.id_off;
  // Zd[0] = M_TT (packed lower, tail rows < 2r; the rest unused) and the identity
  for (int e = lane; e < kTorZE; e += 32) {
    int i, jj;
    tor_tri_ij(e, i, jj);
    zd[e] = (i < 2 * r) ? tor_m(Oc, dim, tor_tail_g(i, q, k), tor_tail_g(jj, q, k)) : 0.0;
    zid[e] = i == jj ? 1.0 : 0.0;
  }
  if (lane == 0) detat[0] = 1.0;
  int zi[2], zj[2];  // this lane's packed Zd entries (lane, lane + 32)
#pragma unroll
  for (int h = 0; h < 2; ++h) tor_tri_ij(lane + 32 * h < kTorZE ? lane + 32 * h : 0, zi[h], zj[h]);
  __syncwarp();
  bool ok = true;
  int count = 0;
  for (int j = 0; j < g; ++j)
    if ((pat >> j) & 1u) {
      ok = tor_w_append(Oc, k, q, r, j, count, col, inv, zd, detat, gidx, lane, zi, zj) && ok;
      ++count;
    }
  const int pc = count;
  double sum = 0.0, sabs = 0.0, srad = 0.0;
  const int rp = q - g;
  const uint64_t nT = 1ull << rp;
  for (uint64_t Tm = 0; Tm < nT; ++Tm) {
    if (Tm) {
      // counter bit b <-> prefix mode g + rp - 1 - b (lowest bit = last prefix mode)
      const int z = __ffsll((long long)Tm) - 1;
      const int jz = g + rp - 1 - z;
      count = pc + __popcll((long long)(Tm >> (z + 1)));
      ok = tor_w_append(Oc, k, q, r, jz, count, col, inv, zd, detat, gidx, lane, zi, zj) && ok;
      ++count;
    }
    int m = 0;
    const double t = tor_w_leaf(zd + count * kTorZE, zid, r, count, k, detat[count], lane, ok, m);
    if (CERT) {
      // ball butterfly: the value operations are those of warp_sum_d
      double v = t;
      double rr = (t != 0.0) ? ru_add(ru_mul(fabs(t), rho[m]), kUfl) : 0.0;
#pragma unroll
      for (int mm = 16; mm > 0; mm >>= 1) {
        const double ov = shfl_xor_d(v, mm), orr = shfl_xor_d(rr, mm);
        v += ov;
        rr = ru_add(ru_add(rr, orr), ru_mul(kUc, fabs(v)));
      }
      sum += v;
      srad = ru_add(ru_add(srad, rr), ru_mul(kUc, fabs(sum)));
    } else {
      sum += warp_sum_d(t);
      if (KAPPA) sabs += warp_sum_d(fabs(t));
    }
  }
  total = sum;
  aux = CERT ? srad : sabs;
  return __all_sync(0xffffffffu, ok);
}

}  // namespace gbsb
