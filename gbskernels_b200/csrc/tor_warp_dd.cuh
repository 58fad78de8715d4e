// tor_warp_dd.cuh -- double-double torontonian: the warp-cooperative prefix-Cholesky
// walk of tor_warp.cuh carried in double-word arithmetic (gbs_common.cuh dd_*), with
// a 16-subset tail (r = min(k, 4) modes, 8 x 8 factors per lane in registers).
//
// Same algorithm and decomposition as the binary64 walk (reference:
// core/tor_recursive.cu:41-115 and its double-double twin core/torontonian_dd.cu:48-88
// for the dd tier): the prefix modes are walked in binary-counter order by the whole
// warp, each append computing the two new factor rows and W rows by one forward
// substitution and updating the tail Schur complement Zd of the new depth; at every
// prefix leaf lanes 0..15 factor Z restricted to their tail subset (rows of excluded
// modes read from a packed identity, pivot reciprocal 0) and the signed terms
// 1 / sqrt(det(M_S) det(Z_T')) are summed by a butterfly in double-word.
// Pivot reciprocals 1 / sqrt(s) are one Newton step from the binary64 rsqrt seed:
// y = y0 + y0 (1 - s y0^2) / 2 in double-word.  The diagonal 1 - O_ii is formed
// exactly (TwoSum), so M enters the walk without rounding.
//
// Certified double-double tier (kTierCertDD): the same walk (the value equals the
// dd tier's bit for bit) with the a-posteriori radius of tor_warp.cuh re-derived for
// double-word operations.  Per-operation relative error bounds (u = 2^-53):
//   dd_add (the accurate double-word sum, Joldes-Muller-Popescu 2017, Alg. 6): 3u^2;
//   dd_mul (TwoProd of the heads, both cross terms by FMA into the tail, Fast2Sum):
//     error = xl*yh*d3 + (xh*yl + e1)(d2 + d3 + d2*d3) - xl*yl, at most 6u^2 + O(u^3)
//     relative (|xl| <= u|xh|, |yl| <= u|yh|, |e1| <= u|xh*yh|); charged 7u^2;
//   dd_mul_d: 2u^2 + O(u^3), charged 3u^2;
//   dd_rsqrt: the Newton step leaves (3/2) e0^2 of the seed's relative error e0 <= 4u
//     (rsqrt taken as 2 ulp) plus the roundings of its four operations: charged 40u^2.
// Every factor entry is an inner product of <= m terms, each a dd_mul and a dd_add,
// plus one scaling; the diagonal carries (1 + 40u^2)^2 from the pivot reciprocal:
// gamma_{2m+16}(7u^2) covers all of it.  With sigma from the same binary64 eigenvalue
// proof, rho_m follows as in tor_warp.cuh but evaluated as small quantities (1 + rho
// is not representable in binary64): tor_cert_rho_dd.
#pragma once

#include "gbs_common.cuh"
#include "tor_warp.cuh"

namespace gbsb {

constexpr int kTorTailDD = 4;                             // tail modes (16 subsets)
constexpr int kTorTDdd = 2 * kTorTailDD;                  // 8 tail rows
constexpr int kTorZEdd = kTorTDdd * (kTorTDdd + 1) / 2;  // 36 packed entries

struct TorDLayout {
  int col_off, inv_off, zd_off, det_off, gidx_off, id_off, rho_off, total;  // in doubles
};

// column u holds (rows - u) prefix slots + 8 tail slots, each a double-word
__host__ __device__ inline int tor_col_base_dd(int u, int rows) { return u * (rows + kTorTDdd) - (u * (u - 1)) / 2; }

__host__ __device__ inline TorDLayout tor_d_layout(int kmax, bool cert = false) {
  TorDLayout Lw;
  const int q = kmax > kTorTailDD ? kmax - kTorTailDD : 0;
  const int rows = 2 * q;
  Lw.col_off = 0;
  Lw.inv_off = Lw.col_off + 2 * (tor_col_base_dd(rows, rows) + 1);
  Lw.zd_off = Lw.inv_off + 2 * (rows + 1);
  Lw.det_off = Lw.zd_off + 2 * (q + 1) * kTorZEdd;
  if (cert) {  // the eigenvalue proof factors a packed 2k x 2k matrix (+ 2k scalings) here
    const int need = (2 * kmax) * (2 * kmax + 1) / 2 + 2 * kmax + 8;
    if (Lw.det_off < need) Lw.det_off = (need + 1) & ~1;
  }
  Lw.gidx_off = Lw.det_off + 2 * (q + 2);
  Lw.id_off = (Lw.gidx_off + (rows + 2) / 2 + 2) & ~1;  // 16-byte aligned double-words
  Lw.rho_off = Lw.id_off + 2 * kTorZEdd;
  Lw.total = Lw.rho_off + (cert ? 2 * kmax + 2 : 0);
  Lw.total = (Lw.total + 3) & ~3;
  return Lw;
}

// entry of M = I - O as a double-word (the diagonal 1 - O_ii exact by TwoSum)
__device__ __forceinline__ dd tor_m_dd(const double* __restrict__ Oc, int dim, int a, int b) {
  const double o = Oc[2 * (a * dim + b)];
  return a == b ? dd_add_d(dd_make(1.0), -o) : dd_make(-o);
}

__device__ __forceinline__ dd ld_dd(const double* p) {
  const double2 v = *reinterpret_cast<const double2*>(p);
  return dd{v.x, v.y};
}
__device__ __forceinline__ void st_dd(double* p, dd v) { *reinterpret_cast<double2*>(p) = make_double2(v.hi, v.lo); }
__device__ __forceinline__ dd shfl_dd(dd v, int src) {
  return dd{__shfl_sync(0xffffffffu, v.hi, src), __shfl_sync(0xffffffffu, v.lo, src)};
}
// a - b c
__device__ __forceinline__ dd dd_fms(dd a, dd b, dd c) { return dd_sub(a, dd_mul(b, c)); }
// 1 / sqrt(s), s > 0: binary64 seed, one Newton step in double-word
__device__ __forceinline__ dd dd_rsqrt(dd s) {
  const double y0 = rsqrt(s.hi);
  const dd t = dd_mul_d(dd_mul_d(s, y0), y0);  // s y0^2
  const dd r = dd_sub(dd_make(1.0), t);       // 1 - s y0^2 (small)
  return dd_add(dd_make(y0), dd_mul_d(r, 0.5 * y0));
}
__device__ __forceinline__ dd warp_sum_dd(dd v) {
#pragma unroll
  for (int m = 16; m > 0; m >>= 1) v = dd_add(v, dd{shfl_xor_d(v.hi, m), shfl_xor_d(v.lo, m)});
  return v;
}

__device__ __forceinline__ int tor_tail_g_dd(int jt, int q, int k) {
  return (jt & 1) ? q + (jt >> 1) + k : q + (jt >> 1);
}

// Append prefix mode j as rows R0 = 2c, R1 = 2c + 1 (double-word).  Out of line: the
// walk calls it from three places, and this walk is bound by instruction fetch
// (one copy instead of three measured +17 % on the double-double tier, values
// bit-identical); (zi0, zj0), (zi1, zj1) are the lane's two packed tail entries.
static __device__ __noinline__ bool tor_d_append(const double* __restrict__ Oc, int k, int q, int r, int j, int c,
                                                 double* col, double* inv, double* zd, double* detat, int* gidx,
                                                 int lane, int zi0, int zi1, int zj0, int zj1) {
  const int zi[2] = {zi0, zi1}, zj[2] = {zj0, zj1};
  const int dim = 2 * k;
  const int rows = 2 * q;
  const int R0 = 2 * c, R1 = R0 + 1;
  const int gR0 = j, gR1 = j + k;
  const int nx = R0 + 2 * r;
  if (lane == 0) {
    gidx[R0] = gR0;
    gidx[R1] = gR1;
  }
  dd a[2], b[2];
  int lim[2], off[2];
#pragma unroll
  for (int h = 0; h < 2; ++h) {
    const int x = lane + 32 * h;
    a[h] = dd_make(0.0);
    b[h] = dd_make(0.0);
    lim[h] = x < R0 ? x : (x < nx ? R0 : 0);
    off[h] = x < R0 ? x : rows + (x - R0);
    if (x < R0) {
      const int gc = gidx[x];
      a[h] = tor_m_dd(Oc, dim, gR0, gc);
      b[h] = tor_m_dd(Oc, dim, gR1, gc);
    } else if (x < nx) {
      const int gT = tor_tail_g_dd(x - R0, q, k);
      a[h] = tor_m_dd(Oc, dim, gR0, gT);
      b[h] = tor_m_dd(Oc, dim, gR1, gT);
    }
  }
  dd d00 = tor_m_dd(Oc, dim, gR0, gR0), d10 = tor_m_dd(Oc, dim, gR1, gR0);
  dd d11 = tor_m_dd(Oc, dim, gR1, gR1);
  double* cv = col;
  auto step = [&](int v, dd av, dd bv) {
    const dd iv = ld_dd(inv + 2 * v);
    const dd l0 = dd_mul(av, iv), l1 = dd_mul(bv, iv);
    if (lane == (v & 31)) {
      st_dd(cv + 2 * (R0 - v), l0);
      st_dd(cv + 2 * (R1 - v), l1);
    }
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      if (v < lim[h]) {
        const dd e = ld_dd(cv + 2 * (off[h] - v));
        a[h] = dd_fms(a[h], e, l0);
        b[h] = dd_fms(b[h], e, l1);
      }
    }
    d00 = dd_fms(d00, l0, l0);
    d10 = dd_fms(d10, l0, l1);
    d11 = dd_fms(d11, l1, l1);
    cv += 2 * (rows + kTorTDdd - v);
  };
  const int v1 = R0 < 32 ? R0 : 32;
  for (int v = 0; v < v1; ++v) step(v, shfl_dd(a[0], v), shfl_dd(b[0], v));
  for (int v = 32; v < R0; ++v) step(v, shfl_dd(a[1], v & 31), shfl_dd(b[1], v & 31));
  dd s0 = d00;
  bool ok = s0.hi > 0.0;
  if (!ok) s0 = dd_make(1.0);
  const dd i0 = dd_rsqrt(s0);
  const dd l10 = dd_mul(d10, i0);
  dd s1 = dd_fms(d11, l10, l10);
  if (!(s1.hi > 0.0)) {
    ok = false;
    s1 = dd_make(1.0);
  }
  const dd i1 = dd_rsqrt(s1);
  double* c0 = col + 2 * tor_col_base_dd(R0, rows);
  double* c1 = col + 2 * tor_col_base_dd(R1, rows);
#pragma unroll
  for (int h = 0; h < 2; ++h) {
    const int x = lane + 32 * h;
    if (x >= R0 && x < nx) {
      const int jt = x - R0;
      const dd w0 = dd_mul(a[h], i0);
      const dd w1 = dd_mul(dd_fms(b[h], w0, l10), i1);
      st_dd(c0 + 2 * (rows - R0 + jt), w0);
      st_dd(c1 + 2 * (rows - R1 + jt), w1);
    }
  }
  if (lane == 0) {
    st_dd(c0 + 2, l10);
    st_dd(inv + 2 * R0, i0);
    st_dd(inv + 2 * R1, i1);
    st_dd(detat + 2 * (c + 1), dd_mul(dd_mul(ld_dd(detat + 2 * c), s0), s1));
  }
  __syncwarp();
  const double* zs = zd + 2 * c * kTorZEdd;
  double* zt = zd + 2 * (c + 1) * kTorZEdd;
  const double* w0p = c0 + 2 * (rows - R0);
  const double* w1p = c1 + 2 * (rows - R1);
#pragma unroll
  for (int h = 0; h < 2; ++h) {
    const int e = lane + 32 * h;
    if (e < kTorZEdd) {
      dd z = ld_dd(zs + 2 * e);
      if (zi[h] < 2 * r) {
        z = dd_fms(z, ld_dd(w0p + 2 * zi[h]), ld_dd(w0p + 2 * zj[h]));
        z = dd_fms(z, ld_dd(w1p + 2 * zi[h]), ld_dd(w1p + 2 * zj[h]));
      }
      st_dd(zt + 2 * e, z);
    }
  }
  __syncwarp();
  return ok;
}

// Two prefix leaves at once: the half warp h (lane >> 4) factors the tail subsets
// (lane & 15 < 2^r) of the leaf at depth c[h] (Schur complement zc[h], determinant
// detc[h]); with two == false only the first half works.  Returns the signed term.
__device__ __forceinline__ dd tor_d_leaf(const double* zc0, const double* zc1, const double* zid, int r, int c0,
                                         int c1, int k, dd det0, dd det1, bool two, int lane, bool& ok, int& m) {
  dd term = dd_make(0.0);
  m = 0;
  const int half = lane >> 4, sub = lane & 15;
  if ((two || half == 0) && sub < (1 << r)) {
    const double* zc = half ? zc1 : zc0;
    const int c = half ? c1 : c0;
    const dd detc = half ? det1 : det0;
    const int td = 2 * r;
    dd Lz[kTorZEdd];
    dd iv[kTorTDdd];
    dd det = dd_make(1.0);
#pragma unroll
    for (int i = 0; i < kTorTDdd; ++i) {
      const bool in_i = i < td && ((sub >> (i >> 1)) & 1);
      const double* zr = (in_i ? zc : zid) + 2 * (i * (i + 1) / 2);
#pragma unroll
      for (int jj = 0; jj <= i; ++jj) {
        const int e = i * (i + 1) / 2 + jj;
        dd s = ld_dd(zr + 2 * jj);
#pragma unroll
        for (int u = 0; u < jj; ++u) s = dd_fms(s, Lz[i * (i + 1) / 2 + u], Lz[jj * (jj + 1) / 2 + u]);
        if (jj < i) {
          Lz[e] = dd_mul(s, iv[jj]);
        } else {
          if (!(s.hi > 0.0)) {
            ok = false;
            s = dd_make(1.0);
          }
          iv[i] = in_i ? dd_rsqrt(s) : dd_make(0.0);
          det = dd_mul(det, s);
        }
      }
    }
    const int nin = __popc(sub);
    m = 2 * (c + nin);
    const dd t = dd_rsqrt(dd_mul(detc, det));
    term = ((k - c - nin) & 1) ? dd_neg(t) : t;
  }
  return term;
}

// rho_m for m = 0..2k in double-double (see the header): all terms are small, so the
// bound is assembled as small quantities in upward rounding,
//   Up - 1 <= x + y + x y,  x = (gp + m eta) / (2 (1 - m eta)),  y = (m er + er) / (1 - m er - er)
//   1 - Lo <= z/2 + z^2/2 + m er + er,  z = gp + m eta
// (sqrt(1 + w) <= 1 + w/2; sqrt(1 - w) >= 1 - w/2 - w^2/2 for w <= 1/2).
static __device__ __noinline__ void tor_cert_rho_dd(double sigma, double dmin2, int k, double* rho, int lane) {
  const double u2 = 7.0 * kU * kU;
  const double er = 40.0 * kU * kU;
  for (int m = lane; m <= 2 * k; m += 32) {
    double out;
    if (m == 0) {
      out = 0.0;
    } else if (!(sigma > 0.0) || !(dmin2 > 0.0)) {
      out = INFINITY;
    } else {
      const double md = (double)m;
      const double g = gamma_ru(2.0 * md + 16.0, u2);
      double cm = ru_div(g, rd_sub(1.0, g));
      cm = ru_div(cm, __dmul_rd(rd_sub(1.0, kU), rd_sub(1.0, kU)));
      cm = ru_add(cm, ru_div(ru_mul(2.0 * md + 16.0, 16.0 * kUfl), dmin2));
      const double meta = ru_mul(md, ru_div(ru_mul(md, cm), sigma));
      const double gp = gamma_ru(md + 1.0, u2);
      const double mer = ru_add(ru_mul(md, er), er);
      if (!(meta < 0.25) || !(mer < 0.25)) {
        out = INFINITY;
      } else {
        const double z = ru_add(gp, meta);
        const double x = ru_div(z, ru_mul(2.0, rd_sub(1.0, meta)));
        const double y = ru_div(mer, rd_sub(1.0, mer));
        const double up = ru_add(ru_add(x, y), ru_mul(x, y));
        const double lo = ru_add(ru_add(ru_mul(0.5, z), ru_mul(0.5, ru_mul(z, z))), mer);
        out = fmax(up, lo);
      }
    }
    rho[m] = out;
  }
  __syncwarp();
}

// One work item: prefix pattern `pat` over the first g walked modes, then every
// subset of the walked modes [g, q) with its 2^r tail subsets.
template <bool CERT>
static __device__ bool tor_dd_item(const double* __restrict__ Oc, int k, int g, uint32_t pat, double* ws,
                                   const TorDLayout& Lw, const double* rho, int lane, dd& total, double& aux) {
  const int dim = 2 * k;
  const int r = k < kTorTailDD ? k : kTorTailDD;
  const int q = k - r;
  double* col = ws + Lw.col_off;
  double* inv = ws + Lw.inv_off;
  double* zd = ws + Lw.zd_off;
  double* detat = ws + Lw.det_off;
  int* gidx = reinterpret_cast<int*>(ws + Lw.gidx_off);
  double* zid = ws + Lw.id_off;
  for (int e = lane; e < kTorZEdd; e += 32) {
    int i, jj;
    tor_tri_ij(e, i, jj);
    st_dd(zd + 2 * e, (i < 2 * r) ? tor_m_dd(Oc, dim, tor_tail_g_dd(i, q, k), tor_tail_g_dd(jj, q, k)) : dd_make(0.0));
    st_dd(zid + 2 * e, dd_make(i == jj ? 1.0 : 0.0));
  }
  if (lane == 0) st_dd(detat, dd_make(1.0));
  int zi[2], zj[2];
#pragma unroll
  for (int h = 0; h < 2; ++h) tor_tri_ij(lane + 32 * h < kTorZEdd ? lane + 32 * h : 0, zi[h], zj[h]);
  __syncwarp();
  bool ok = true;
  int count = 0;
  for (int j = 0; j < g; ++j)
    if ((pat >> j) & 1u) {
      ok = tor_d_append(Oc, k, q, r, j, count, col, inv, zd, detat, gidx, lane, zi[0], zi[1], zj[0], zj[1]) && ok;
      ++count;
    }
  const int pc = count;
  dd sum = dd_make(0.0);
  double srad = 0.0;
  constexpr double kU2x4 = 4.0 * kU * kU;  // bound of one dd_add, relative, with slack
  const int rp = q - g;
  // The walked modes [g, q) in binary-counter order, the last one (q - 1) as the
  // lowest bit: the leaves come in sibling pairs (q - 1 out, then in).  After the
  // append of q - 1 both siblings' Schur complements and determinants are in shared
  // memory (depths c and c + 1), so one pass factors both, a half warp each (the
  // 16 tail subsets of a leaf fill only half the lanes).  Each term is the one the
  // leaf gives alone; the sum takes them in another order.
  const bool pairs = rp > 0 && r == kTorTailDD;
  const uint64_t nT = 1ull << (pairs ? rp - 1 : rp);
  for (uint64_t Tp = 0; Tp < nT; ++Tp) {
    const uint64_t Tm = pairs ? 2 * Tp : Tp;
    if (Tm) {
      const int z = __ffsll((long long)Tm) - 1;
      const int jz = g + rp - 1 - z;
      count = pc + __popcll((long long)(Tm >> (z + 1)));
      ok = tor_d_append(Oc, k, q, r, jz, count, col, inv, zd, detat, gidx, lane, zi[0], zi[1], zj[0], zj[1]) && ok;
      ++count;
    }
    if (pairs) ok = tor_d_append(Oc, k, q, r, q - 1, count, col, inv, zd, detat, gidx, lane, zi[0], zi[1], zj[0], zj[1]) && ok;
    int m = 0;
    const dd t = tor_d_leaf(zd + 2 * count * kTorZEdd, zd + 2 * (count + 1) * kTorZEdd, zid, r, count, count + 1, k,
                            ld_dd(detat + 2 * count), ld_dd(detat + 2 * (count + 1)), pairs, lane, ok, m);
    if (CERT) {
      // ball butterfly: the value operations are those of warp_sum_dd
      dd v = t;
      double rr = (t.hi != 0.0) ? ru_add(ru_mul(ru_mul(fabs(t.hi), 1.0 + 4.0 * kU), rho[m]), kUfl) : 0.0;
#pragma unroll
      for (int mm = 16; mm > 0; mm >>= 1) {
        const dd ov{shfl_xor_d(v.hi, mm), shfl_xor_d(v.lo, mm)};
        const double orr = shfl_xor_d(rr, mm);
        v = dd_add(v, ov);
        rr = ru_add(ru_add(rr, orr), ru_add(ru_mul(kU2x4, fabs(v.hi)), kUfl));
      }
      sum = dd_add(sum, v);
      srad = ru_add(ru_add(srad, rr), ru_add(ru_mul(kU2x4, fabs(sum.hi)), kUfl));
    } else {
      sum = dd_add(sum, warp_sum_dd(t));
    }
  }
  total = sum;
  aux = srad;
  return __all_sync(0xffffffffu, ok);
}

}  // namespace gbsb
