// k_sieve.cu -- loop hafnians of repeated-row expansions by the finite-difference
// sieve, batched over repetition patterns of one shared base matrix.
//
// lhaf(A[n], gamma[n]) = sum_{v <= n} (-1)^{|v|} prod_i C(n_i, v_i) S_N(x_v) / (N! 2^N),
//   x_v = n - 2v,  S_N(x) = sum_k C(N, 2k) (2k-1)!! (x^T A x)^k (x . gamma)^{N-2k},
// where A[n] repeats row / column i of the M x M base matrix n_i times and puts
// gamma_i on the diagonal of every copy (gamma = 0: the ordinary hafnian of the
// expansion).  Reference: cpu_ref/repeated.py:64-122 (derivation and the v <-> n - v
// symmetry), core/repeated.cu:44-160 (one pattern per thread, caps M <= 32, N <= 64).
//
// B200 mapping (this repository's design):
//   * a pattern's digits are its modes with n_i > 0, the largest n_i on top; the top
//     digit runs over 0..floor(n_top / 2) only (weight 2 below the middle, 1 on it:
//     the v <-> n - v symmetry, exact in binary64 because x -> -x only flips signs);
//   * the sieve terms are walked in REFLECTED MIXED-RADIX GRAY order, so consecutive
//     terms differ in one digit by +-1: with lane i holding digit i, x_i and
//     (A x)_i, a step costs one column of A (A x += d A e_j), two shuffles and the
//     scalar updates sigma^2 += d (2 (Ax)_j + d A_jj), mu += d gamma_j;
//   * one warp per work item of at most kSieveItem consecutive terms (the item's
//     start state is decoded from its Gray index and A x is formed directly, so the
//     incremental updates never run longer than one item); the scalar pairs
//     (sigma^2, mu) and the signed binomial weights of 32 consecutive terms are
//     parked one per lane, then the 32 lanes evaluate S_N at once (Horner in sigma^2
//     with the mu^2 powers alongside, normalisation folded into the coefficients);
//   * item partials are reduced per pattern in item order by a second small kernel:
//     the result is deterministic.
//   * a non-symmetric base matrix enters as its symmetric part (A + A^T) / 2 (x^T A x
//     only sees that part; the incremental update needs it); a symmetric one is
//     unchanged bit for bit.
//
// Certified sieve (CERT; reference counterpart core/repeated.cu:158-340, which
// recomputes every term from scratch): the same walk, so the value is the plain
// sieve's bit for bit, with running radii in upward rounding (u = 2^-53, L1 norms
// |re| + |im| >= |z|): the start state of an item by gamma bounds of its sums; every
// Gray step adds the rounding of its updates (the scalings by +-2 are exact) to the
// radii of (A x)_i, sigma^2 and mu; a parked term's S_N errs by at most
// gamma_{8K+16} B(s~, m~) (Horner and power roundings, coefficient representation)
// plus B(s~, m~) - B(|s|, |mu|) (its inputs' radii), B the polynomial with |cf_k|
// evaluated upward at s~ = |s| + r_s, m~ = |mu| + r_mu; the signed binomial weight
// carries gamma_{3 nd + 8}; sums add u |partial sum| per operation.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "cert.cuh"
#include "gbs_common.cuh"

namespace gbsb {

constexpr int kSieveMaxM = 32;
constexpr int kSieveMaxN = 64;
constexpr int kSieveMaxK = kSieveMaxN / 2;
constexpr long long kSieveMaxItems = 1ll << 26;  // partial storage: 1 GiB

struct SievePattern {
  unsigned long long terms;  // sieve terms walked (top digit halved)
  unsigned long long item_len;
  long long item0;           // first global item of this pattern
  int nd;                    // digits (modes with n > 0); 0 = empty pattern
  int N;                     // photons = sum n
  int mode[kSieveMaxM];      // digit -> base-matrix row (digit 0 changes fastest)
  int reps[kSieveMaxM];      // n of each digit
  int radix[kSieveMaxM];     // n + 1, the top digit floor(n / 2) + 1
  unsigned long long place[kSieveMaxM];  // product of the radices below the digit
  double esym;               // certified: radius of sigma^2 from rounding (A + A^T) / 2 (0 if symmetric)
};

__device__ __forceinline__ cplx shfl_c(cplx v, int src) {
  return mkc(__shfl_sync(0xffffffffu, v.re, src), __shfl_sync(0xffffffffu, v.im, src));
}

// product of v over the warp, fixed butterfly order (every lane gets it)
__device__ __forceinline__ double warp_prod_d(double v) {
#pragma unroll
  for (int m = 16; m > 0; m >>= 1) v *= shfl_xor_d(v, m);
  return v;
}

// S_N(s, mu) with the normalised coefficients cf[k] = C(N,2k)(2k-1)!!/(N! 2^N):
// sum_k cf[k] s^k w^{K-k} (times mu for odd N), w = mu^2, by Horner in s.
__device__ __forceinline__ cplx sieve_sn(cplx s, cplx mu, int N, const double* __restrict__ cf) {
  const int K = N >> 1;
  const cplx w = cmul(mu, mu);
  cplx h = mkc(cf[K], 0.0);
  cplx wk = w;
  for (int k = K - 1; k >= 0; --k) {
    h = cadd(cmul(h, s), cscale(wk, cf[k]));
    wk = cmul(wk, w);
  }
  return (N & 1) ? cmul(h, mu) : h;
}

// B(s, m) = sum_k |cf[k]| s^k m^{2(K-k)} (times m for odd N) for s, m >= 0, by
// Horner in upward (UP) or downward rounding.
template <bool UP>
__device__ __forceinline__ double sieve_bpoly(double s, double m, int N, const double* __restrict__ cf) {
  const int K = N >> 1;
  auto mul = [](double a, double b) { return UP ? ru_mul(a, b) : rd_mul(a, b); };
  auto add = [](double a, double b) { return UP ? ru_add(a, b) : rd_add(a, b); };
  const double w = mul(m, m);
  double h = fabs(cf[K]);
  double wk = w;
  for (int k = K - 1; k >= 0; --k) {
    h = add(mul(h, s), mul(wk, fabs(cf[k])));
    wk = mul(wk, w);
  }
  return (N & 1) ? mul(h, m) : h;
}
__device__ __forceinline__ double mag1_ru(cplx z) { return ru_add(fabs(z.re), fabs(z.im)); }

template <bool CERT>
__global__ void __launch_bounds__(128) sieve_kernel(const double* __restrict__ A, const double* __restrict__ gamma,
                                                    int M, const SievePattern* __restrict__ pats, int npat,
                                                    long long nitems, const double* __restrict__ coef,
                                                    const double* __restrict__ binom, double* __restrict__ part,
                                                    double* __restrict__ part_r) {
  const int lane = threadIdx.x & 31;
  const long long warps = (long long)gridDim.x * (blockDim.x >> 5);
  for (long long it = (long long)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); it < nitems; it += warps) {
    // the pattern owning item `it` (patterns are in item order)
    int lo = 0, hi = npat - 1;
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (pats[mid].item0 <= it) lo = mid;
      else hi = mid - 1;
    }
    const SievePattern& P = pats[lo];
    const int nd = P.nd, N = P.N;
    const double* cf = coef + (size_t)N * (kSieveMaxK + 1);
    const unsigned long long t0 = (unsigned long long)(it - P.item0) * P.item_len;
    const unsigned long long t1 = min(t0 + P.item_len, P.terms);
    // ---- start state at Gray index t0
    const bool act = lane < nd;
    int mi = 0, ni = 0, ri = 1, b = 0, par = 0, g = 0;
    if (act) {
      mi = P.mode[lane];
      ni = P.reps[lane];
      ri = P.radix[lane];
      const unsigned long long q = t0 / P.place[lane];
      b = (int)(q % (unsigned long long)ri);
      par = (lane == nd - 1) ? 0 : (int)((q / (unsigned long long)ri) & 1ull);
      g = par ? ri - 1 - b : b;
    }
    double x = act ? (double)(ni - 2 * g) : 0.0;
    cplx ax = mkc(0.0, 0.0);
    double max_ = 0.0;  // certified: sum_d |A[i][d]| |x_d|
    for (int d = 0; d < nd; ++d) {
      const int md = __shfl_sync(0xffffffffu, mi, d);
      const double xd = __shfl_sync(0xffffffffu, x, d);
      if (act) {
        const cplx a = ld_c(A + 2 * ((size_t)mi * M + md));
        ax = cadd(ax, cscale(a, xd));
        if constexpr (CERT) max_ = ru_add(max_, ru_mul(mag1_ru(a), fabs(xd)));
      }
    }
    cplx sig2 = warp_sum_c(cscale(ax, x));
    cplx mu = warp_sum_c(act ? cscale(ld_c(gamma + 2 * mi), x) : mkc(0.0, 0.0));
    // certified radii (L1) of (A x)_i, sigma^2 and mu at the item start
    double rax = 0.0, rs = 0.0, rm = 0.0;
    if constexpr (CERT) {
      const double g6 = gamma_ru(6.0, kU);
      if (act) rax = ru_add(ru_mul(gamma_ru((double)nd, kU), max_), (double)nd * kUfl);
      rs = warp_sum_ru(act ? ru_add(ru_mul(g6, ru_mul(fabs(x), mag1_ru(ax))), ru_mul(fabs(x), rax)) : 0.0);
      rs = ru_add(rs, 64.0 * kUfl);
      rm = warp_sum_ru(act ? ru_mul(g6, ru_mul(fabs(x), mag1_ru(ld_c(gamma + 2 * mi)))) : 0.0);
      rm = ru_add(rm, 64.0 * kUfl);
    }
    const double esym = CERT ? P.esym : 0.0;
    const int K = N >> 1;
    const double ghorn = CERT ? gamma_ru(8.0 * K + 16.0, kU) : 0.0;
    const double crel = CERT ? gamma_ru(3.0 * nd + 8.0, kU) : 0.0;
    double cd = act ? binom[ni * (kSieveMaxN + 1) + g] : 1.0;
    double c0 = __shfl_sync(0xffffffffu, cd, 0);
    double crest = warp_prod_d(lane == 0 ? 1.0 : cd);
    int vpar = __popc(__ballot_sync(0xffffffffu, act && (g & 1)));  // parity of |v| below
    vpar &= 1;
    int gtop = __shfl_sync(0xffffffffu, g, nd - 1), ntop = __shfl_sync(0xffffffffu, ni, nd - 1);
    // ---- walk
    cplx ps = mkc(0.0, 0.0), pm = mkc(0.0, 0.0);  // this lane's parked term
    double pc = 0.0;
    double prs = 0.0, prm = 0.0;  // certified: the parked radii
    cplx acc = mkc(0.0, 0.0);
    double racc = 0.0;            // certified: radius of this lane's acc
    for (unsigned long long t = t0; t < t1; ++t) {
      const int slot = (int)((t - t0) & 31ull);
      const double wgt = (2 * gtop < ntop) ? 2.0 : 1.0;
      if (lane == slot) {
        ps = sig2;
        pm = mu;
        pc = (vpar ? -wgt : wgt) * c0 * crest;
        if constexpr (CERT) {
          prs = ru_add(rs, esym);
          prm = rm;
        }
      }
      if (slot == 31 || t + 1 == t1) {
        if (lane <= slot) {
          const cplx sn = sieve_sn(ps, pm, N, cf);
          const cplx term = cscale(sn, pc);
          acc = cadd(acc, term);
          if constexpr (CERT) {
            const double sa = mag1_ru(ps), ma = mag1_ru(pm);
            const double bup = sieve_bpoly<true>(ru_add(sa, prs), ru_add(ma, prm), N, cf);
            const double bdn = sieve_bpoly<false>(sa, ma, N, cf);
            double esn = ru_add(ru_mul(ghorn, bup), ru_add(bup, -bdn));
            esn = ru_add(esn, (double)(4 * K + 8) * kUfl);
            double et = ru_mul(fabs(pc), esn);
            et = ru_add(et, ru_mul(ru_add(crel, kU), ru_mul(fabs(pc), mag1_ru(sn))));
            racc = ru_add(ru_add(racc, et), ru_add(ru_mul(kU, mag1_ru(acc)), 2.0 * kUfl));
          }
        }
      }
      if (t + 1 == t1) break;
      // one reflected Gray step: digit j moves by dir
      const unsigned cand = __ballot_sync(0xffffffffu, act && b < ri - 1);
      const int j = __ffs(cand) - 1;
      const int dir = ((__ballot_sync(0xffffffffu, par != 0) >> j) & 1u) ? -1 : 1;
      if (lane < j) {
        b = 0;
        par ^= 1;
      } else if (lane == j) {
        b += 1;
        g += dir;
        x = (double)(ni - 2 * g);
        cd = binom[ni * (kSieveMaxN + 1) + g];
      }
      const double dlt = -2.0 * dir;  // change of x_j
      const int mj = __shfl_sync(0xffffffffu, mi, j);
      const cplx axj = shfl_c(ax, j);
      const cplx ajj = ld_c(A + 2 * ((size_t)mj * M + mj));
      const cplx inner = cadd(cscale(axj, 2.0), cscale(ajj, dlt));
      sig2 = cadd(sig2, cscale(inner, dlt));
      mu = cadd(mu, cscale(ld_c(gamma + 2 * mj), dlt));
      if constexpr (CERT) {
        // the scalings by 2 and +-2 are exact; one rounding per complex sum
        const double raxj = __shfl_sync(0xffffffffu, rax, j);
        rs = ru_add(rs, ru_mul(2.0, ru_add(ru_mul(2.0, raxj), ru_add(ru_mul(kU, mag1_ru(inner)), kUfl))));
        rs = ru_add(rs, ru_add(ru_mul(kU, mag1_ru(sig2)), kUfl));
        rm = ru_add(rm, ru_add(ru_mul(kU, mag1_ru(mu)), kUfl));
      }
      if (act) {
        ax = cadd(ax, cscale(ld_c(A + 2 * ((size_t)mj * M + mi)), dlt));
        if constexpr (CERT) rax = ru_add(rax, ru_add(ru_mul(kU, mag1_ru(ax)), kUfl));
      }
      vpar ^= 1;
      if (j == 0) {
        c0 = __shfl_sync(0xffffffffu, cd, 0);
      } else {
        crest = warp_prod_d(lane == 0 ? 1.0 : cd);
        if (j == nd - 1) gtop = __shfl_sync(0xffffffffu, g, nd - 1);
      }
    }
    double rbut = 0.0;
    if constexpr (CERT) rbut = ru_add(warp_sum_ru(racc), ru_mul(gamma_ru(5.0, kU), warp_sum_ru(mag1_ru(acc))));
    acc = warp_sum_c(acc);
    if (lane == 0) {
      part[2 * it] = acc.re;
      part[2 * it + 1] = acc.im;
      if constexpr (CERT) part_r[it] = ru_add(rbut, 32.0 * kUfl);
    }
  }
}

// One warp per pattern: the item partials in item order (lane-strided, then a fixed
// butterfly); empty patterns give 1.
template <bool CERT>
__global__ void __launch_bounds__(128) sieve_reduce_kernel(const SievePattern* __restrict__ pats, int npat,
                                                           const double* __restrict__ part,
                                                           const double* __restrict__ part_r, double* __restrict__ out,
                                                           double* __restrict__ out_r) {
  const int lane = threadIdx.x & 31;
  const int p = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  if (p >= npat) return;
  const SievePattern& P = pats[p];
  if (P.nd == 0) {
    if (lane == 0) {
      out[2 * p] = 1.0;
      out[2 * p + 1] = 0.0;
      if constexpr (CERT) out_r[p] = 0.0;
    }
    return;
  }
  const long long nit = (long long)((P.terms + P.item_len - 1) / P.item_len);
  cplx s = mkc(0.0, 0.0);
  double r = 0.0, mg = 0.0;
  for (long long k = lane; k < nit; k += 32) {
    const cplx v = ld_c(part + 2 * (P.item0 + k));
    s = cadd(s, v);
    if constexpr (CERT) {
      r = ru_add(r, part_r[P.item0 + k]);
      mg = ru_add(mg, mag1_ru(v));
    }
  }
  if constexpr (CERT) {
    // lane sums of ceil(nit / 32) partials, then the butterfly: gamma_{n/32 + 5}
    const double gs = gamma_ru((double)((nit + 31) / 32 + 5), kU);
    r = ru_add(warp_sum_ru(r), ru_mul(gs, warp_sum_ru(mg)));
  }
  s = warp_sum_c(s);
  if (lane == 0) {
    out[2 * p] = s.re;
    out[2 * p + 1] = s.im;
    if constexpr (CERT) out_r[p] = ru_add(r, 32.0 * kUfl);
  }
}

namespace {
thread_local std::string t_sieve_err;
int sieve_fail(int code, const std::string& msg) {
  t_sieve_err = msg;
  return code;
}

struct SieveTables {
  std::vector<double> coef, binom;
};
const SieveTables& tables() {
  static SieveTables T = [] {
    SieveTables t;
    t.coef.assign((size_t)(kSieveMaxN + 1) * (kSieveMaxK + 1), 0.0);
    t.binom.assign((size_t)(kSieveMaxN + 1) * (kSieveMaxN + 1), 0.0);
    for (int n = 0; n <= kSieveMaxN; ++n)
      for (int k = 0; k <= n; ++k) {
        long double c = 1.0L;
        for (int u = 1; u <= k; ++u) c = c * (long double)(n - k + u) / (long double)u;
        t.binom[(size_t)n * (kSieveMaxN + 1) + k] = (double)c;
      }
    for (int N = 0; N <= kSieveMaxN; ++N) {
      // C(N, 2k) (2k-1)!! / (N! 2^N) in extended precision
      long double norm = 1.0L;
      for (int u = 2; u <= N; ++u) norm *= (long double)u;
      norm = ldexpl(norm, N);
      for (int k = 0; 2 * k <= N; ++k) {
        long double c = 1.0L;
        for (int u = 1; u <= 2 * k; ++u) c = c * (long double)(N - 2 * k + u) / (long double)u;
        for (int u = 2 * k - 1; u > 0; u -= 2) c *= (long double)u;
        t.coef[(size_t)N * (kSieveMaxK + 1) + k] = (double)(c / norm);
      }
    }
    return t;
  }();
  return T;
}
}  // namespace

}  // namespace gbsb

using namespace gbsb;

namespace {
// Plain (bound == nullptr) or certified evaluation of a batch of patterns.
// Device buffers of the sieve, kept per device between calls and grown only when a
// call needs more (the tables are uploaded once per device).  Allocating and
// freeing them per call cost more host time than the sieve kernels of a
// 4096-pattern batch (cudaFree synchronises the device).  Calls hold g_sieve_mu.
struct SieveBufs {
  double *A = nullptr, *g = nullptr, *coef = nullptr, *bin = nullptr, *part = nullptr, *out = nullptr,
         *part_r = nullptr, *out_r = nullptr;
  SievePattern* pats = nullptr;
  size_t cap_A = 0, cap_g = 0, cap_part = 0, cap_out = 0, cap_pats = 0, cap_part_r = 0, cap_out_r = 0;
};
constexpr int kSieveDevs = 64;
SieveBufs g_sieve[kSieveDevs];
std::mutex g_sieve_mu;

template <typename T>
cudaError_t sieve_grow(T** p, size_t* cap, size_t n) {
  if (n <= *cap) return cudaSuccess;
  if (*p) cudaFree(*p);
  *p = nullptr;
  *cap = 0;
  const cudaError_t e = cudaMalloc(p, sizeof(T) * n);
  if (e == cudaSuccess) *cap = n;
  return e;
}

int sieve_run(const double* A_in, const double* gamma, int M, const int* reps, int batch, double* out,
              double* bound) {
  const bool cert = bound != nullptr;
  if (batch < 0 || M < 0) return sieve_fail((int)cudaErrorInvalidValue, "lhaf_repeated: negative size");
  if (batch == 0) return 0;
  if (!A_in || !reps || !out) return sieve_fail((int)cudaErrorInvalidValue, "lhaf_repeated: null pointer");
  if (M > kSieveMaxM) return sieve_fail((int)cudaErrorInvalidValue, "lhaf_repeated: M above the cap 32");
  if (cert) {
    for (size_t k = 0; k < 2ull * M * M; ++k)
      if (!std::isfinite(A_in[k]))
        return sieve_fail((int)cudaErrorInvalidValue, "certified lhaf_repeated requires finite input");
    if (gamma)
      for (size_t k = 0; k < 2ull * M; ++k)
        if (!std::isfinite(gamma[k]))
          return sieve_fail((int)cudaErrorInvalidValue, "certified lhaf_repeated requires finite input");
  }
  // x^T A x sees only the symmetric part: (A + A^T) / 2, bit-identical to A when
  // A is symmetric (a + a = 2a and the halving are exact)
  std::vector<double> As(2 * (size_t)std::max(M * M, 1), 0.0);
  bool sym = true;
  for (int i = 0; i < M; ++i)
    for (int j = 0; j < M; ++j)
      for (int c = 0; c < 2; ++c) {
        const double a = A_in[2 * ((size_t)i * M + j) + c], b = A_in[2 * ((size_t)j * M + i) + c];
        if (a != b) sym = false;
        As[2 * ((size_t)i * M + j) + c] = (a + b) * 0.5;
      }
  const double* A = As.data();
  const SieveTables& T = tables();
  std::vector<SievePattern> pats((size_t)batch);
  long long items = 0;
  for (int p = 0; p < batch; ++p) {
    SievePattern P{};
    const int* n = reps + (size_t)p * M;
    std::vector<int> modes;
    double terms_full = 1.0;
    for (int i = 0; i < M; ++i) {
      if (n[i] < 0) return sieve_fail((int)cudaErrorInvalidValue, "lhaf_repeated: reps must be non-negative");
      if (n[i] > 0) modes.push_back(i);
      P.N += n[i];
      terms_full *= (double)(n[i] + 1);
    }
    if (P.N > kSieveMaxN) return sieve_fail((int)cudaErrorInvalidValue, "lhaf_repeated: N = sum(reps) above the cap 64");
    if (terms_full > 1.099511627776e12)
      return sieve_fail((int)cudaErrorInvalidValue, "lhaf_repeated: prod(n_i + 1) above the cap 2^40");
    // digits: ascending n (digit 0 fastest), the largest n on top
    std::stable_sort(modes.begin(), modes.end(), [&](int a, int b) { return n[a] < n[b]; });
    P.nd = (int)modes.size();
    unsigned long long place = 1;
    for (int d = 0; d < P.nd; ++d) {
      P.mode[d] = modes[d];
      P.reps[d] = n[modes[d]];
      P.radix[d] = d == P.nd - 1 ? n[modes[d]] / 2 + 1 : n[modes[d]] + 1;
      P.place[d] = place;
      place *= (unsigned long long)P.radix[d];
    }
    P.terms = P.nd ? place : 0;
    // items of 256 terms; longer patterns get longer items (at most 2^20 per pattern)
    unsigned long long len = 256;
    while (P.terms > len * (1ull << 20)) len <<= 1;
    P.item_len = len;
    P.item0 = items;
    items += (long long)((P.terms + len - 1) / len);
    if (items > kSieveMaxItems)
      return sieve_fail((int)cudaErrorInvalidValue, "lhaf_repeated: batch too large for one call (split it)");
    // certified, non-symmetric A: |x^T (A^s - (A + A^T)/2) x| <= u sum n_i n_j |A^s_ij|
    // (one rounding per entry of the symmetric part), charged as 2.25 u
    P.esym = 0.0;
    if (cert && !sym) {
      long double e = 0.0L;
      for (int i = 0; i < M; ++i)
        for (int j = 0; j < M; ++j)
          e += (long double)n[i] * n[j] *
               (std::fabs(As[2 * ((size_t)i * M + j)]) + std::fabs(As[2 * ((size_t)i * M + j) + 1]));
      P.esym = std::nextafter((double)(e * 2.5e-16L), INFINITY);
    }
    pats[p] = P;
  }
  std::vector<double> g0;
  if (!gamma) {
    g0.assign(2 * (size_t)std::max(M, 1), 0.0);
    gamma = g0.data();
  }
  std::lock_guard<std::mutex> lk(g_sieve_mu);
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess || dev < 0 || dev >= kSieveDevs)
    return sieve_fail(e != cudaSuccess ? (int)e : (int)cudaErrorInvalidDevice, "lhaf_repeated: no usable device");
  SieveBufs& Bf = g_sieve[dev];
  if (Bf.coef) {
    // a device reset (cudaDeviceReset) since the last call frees every allocation:
    // the cached pointers then no longer name device memory, and are dropped
    cudaPointerAttributes pa{};
    if (cudaPointerGetAttributes(&pa, Bf.coef) != cudaSuccess || pa.type != cudaMemoryTypeDevice) {
      cudaGetLastError();
      Bf = SieveBufs{};
    }
  }
  if (!Bf.coef) {  // the tables, once per device
    e = cudaMalloc(&Bf.coef, sizeof(double) * T.coef.size());
    if (e == cudaSuccess) e = cudaMalloc(&Bf.bin, sizeof(double) * T.binom.size());
    if (e == cudaSuccess)
      e = cudaMemcpy(Bf.coef, T.coef.data(), sizeof(double) * T.coef.size(), cudaMemcpyHostToDevice);
    if (e == cudaSuccess)
      e = cudaMemcpy(Bf.bin, T.binom.data(), sizeof(double) * T.binom.size(), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) {
      if (Bf.coef) cudaFree(Bf.coef);
      if (Bf.bin) cudaFree(Bf.bin);
      Bf.coef = Bf.bin = nullptr;
    }
  }
  if (e == cudaSuccess) e = sieve_grow(&Bf.A, &Bf.cap_A, 2 * (size_t)std::max(M * M, 1));
  if (e == cudaSuccess) e = sieve_grow(&Bf.g, &Bf.cap_g, 2 * (size_t)std::max(M, 1));
  if (e == cudaSuccess) e = sieve_grow(&Bf.part, &Bf.cap_part, 2 * (size_t)std::max(items, 1ll));
  if (e == cudaSuccess) e = sieve_grow(&Bf.out, &Bf.cap_out, 2 * (size_t)batch);
  if (e == cudaSuccess) e = sieve_grow(&Bf.pats, &Bf.cap_pats, (size_t)batch);
  if (e == cudaSuccess && cert) e = sieve_grow(&Bf.part_r, &Bf.cap_part_r, (size_t)std::max(items, 1ll));
  if (e == cudaSuccess && cert) e = sieve_grow(&Bf.out_r, &Bf.cap_out_r, (size_t)batch);
  double *dA = Bf.A, *dg = Bf.g, *dcoef = Bf.coef, *dbin = Bf.bin, *dpart = Bf.part, *dout = Bf.out;
  double *dpart_r = cert ? Bf.part_r : nullptr, *dout_r = cert ? Bf.out_r : nullptr;
  SievePattern* dpats = Bf.pats;
  if (e == cudaSuccess && M > 0) e = cudaMemcpy(dA, A, sizeof(double) * 2 * M * M, cudaMemcpyHostToDevice);
  if (e == cudaSuccess && M > 0) e = cudaMemcpy(dg, gamma, sizeof(double) * 2 * M, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(dpats, pats.data(), sizeof(SievePattern) * batch, cudaMemcpyHostToDevice);
  if (e == cudaSuccess && items > 0) {
    int sms = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const long long want = (items + 3) / 4;
    const int grid = (int)std::max(1ll, std::min<long long>(want, (long long)sms * 16));
    if (cert) sieve_kernel<true><<<grid, 128>>>(dA, dg, M, dpats, batch, items, dcoef, dbin, dpart, dpart_r);
    else sieve_kernel<false><<<grid, 128>>>(dA, dg, M, dpats, batch, items, dcoef, dbin, dpart, nullptr);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) {
    if (cert) sieve_reduce_kernel<true><<<(batch + 3) / 4, 128>>>(dpats, batch, dpart, dpart_r, dout, dout_r);
    else sieve_reduce_kernel<false><<<(batch + 3) / 4, 128>>>(dpats, batch, dpart, nullptr, dout, nullptr);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaMemcpy(out, dout, sizeof(double) * 2 * batch, cudaMemcpyDeviceToHost);
  if (e == cudaSuccess && cert) e = cudaMemcpy(bound, dout_r, sizeof(double) * batch, cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) return sieve_fail((int)e, std::string("lhaf_repeated: ") + cudaGetErrorString(e));
  if (cert)
    for (int p = 0; p < batch; ++p) {
      // the value is returned in binary64 as computed; a non-finite value or bound
      // is a refusal (NaN, +inf)
      if (!std::isfinite(out[2 * p]) || !std::isfinite(out[2 * p + 1]) || !std::isfinite(bound[p])) {
        out[2 * p] = out[2 * p + 1] = NAN;
        bound[p] = INFINITY;
      }
    }
  return 0;
}
}  // namespace

extern "C" {

// Loop hafnians of the M x M base matrix A (complex, row-major) repeated by each
// row of `reps` (batch x M non-negative counts), loop weights gamma (M complex, NULL =
// zeros: ordinary hafnians of the expansions).  Caps as the reference: M <= 32,
// N = sum(reps row) <= 64, prod(n_i + 1) <= 2^40.
int gbs_lhaf_repeated_host(const double* A, const double* gamma, int M, const int* reps, int batch, double* out) {
  return sieve_run(A, gamma, M, reps, batch, out, nullptr);
}

// Certified: the same values bit for bit and a rigorous bound per pattern.
int gbs_lhaf_repeated_cert_host(const double* A, const double* gamma, int M, const int* reps, int batch, double* out,
                                double* bound) {
  if (batch > 0 && !bound) return sieve_fail((int)cudaErrorInvalidValue, "lhaf_repeated: null bound buffer");
  return sieve_run(A, gamma, M, reps, batch, out, bound ? bound : nullptr);
}

const char* gbs_lhaf_repeated_last_error(void) { return t_sieve_err.c_str(); }

}  // extern "C"
