// gbs_oracle.cpp -- CPU ORACLE (test infrastructure only; never shipped, never timed
// as the product).  A plain restatement of the reference's four matrix functions,
// templated on the real type so the SAME algorithm runs in IEEE binary64 (the
// fp64-tier twin) and in IEEE binary128 (`__float128`, 113-bit significand: the
// high-precision pin for sizes where an mpmath evaluation is out of reach).
//
// Algorithms restated (reference file:line):
//   * permanent, Glynn/BB-FG Gray-code walk ....... cpu_ref/permanent.py:108-139,
//                                                   core/permanent.cu:30-76
//   * hafnian, power trace (diagonal zeroed) ....... cpu_ref/hafnian.py:68-129
//   * loop hafnian, power trace + loop term ........ cpu_ref/loop_hafnian.py:65-108
//     (odd N augmented by A (+) [1] as gbskernels/__init__.py:190-200)
//   * torontonian, recursive prefix Cholesky (real)  core/tor_recursive.cu:41-115,
//                                                   cpu_ref/tor_recursive.py:46-100
//   * torontonian, per-subset determinant (complex)  cpu_ref/torontonian.py:48-64
//   * loop hafnian of a repeated-row expansion,
//     finite-difference sieve ....................... cpu_ref/repeated.py:64-122
//   * sum|term| indicators for precision="auto" ..... cpu_ref/diagnostics.py:40-170,
//                                                   core/permanent.cu:94-130
//
// Complex matrices are passed as interleaved (re, im) binary64 pairs, row-major,
// i.e. numpy complex128 memory.  Every result is returned as a pair (hi, lo) per
// component so a binary128 result survives the trip to numpy at ~2^-106.
//
// Build: oracle/Makefile (g++ -O2 -shared, libquadmath for binary128 sqrt).

#include <quadmath.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

namespace {

template <class T> struct Cx {
  T re, im;
};
template <class T> inline Cx<T> cadd(Cx<T> a, Cx<T> b) { return {a.re + b.re, a.im + b.im}; }
template <class T> inline Cx<T> csub(Cx<T> a, Cx<T> b) { return {a.re - b.re, a.im - b.im}; }
template <class T> inline Cx<T> cmul(Cx<T> a, Cx<T> b) {
  return {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re};
}
template <class T> inline Cx<T> cscale(Cx<T> a, T s) { return {a.re * s, a.im * s}; }

inline double to_d(double x) { return x; }
inline double to_d(__float128 x) { return (double)x; }
inline double tabs(double x) { return std::fabs(x); }
inline __float128 tabs(__float128 x) { return fabsq(x); }
inline double tsqrt(double x) { return std::sqrt(x); }
inline __float128 tsqrt(__float128 x) { return sqrtq(x); }
template <class T> inline double cabs_d(Cx<T> a) { return std::hypot(to_d(a.re), to_d(a.im)); }
template <class T> inline T cabs_t(Cx<T> a) { return tsqrt(a.re * a.re + a.im * a.im); }

// Principal complex square root, the branch numpy's sqrt(complex) takes.
template <class T> Cx<T> csqrt_principal(Cx<T> z) {
  T r = cabs_t(z);
  if (r == T(0)) return {T(0), T(0)};
  T a = tsqrt((r + tabs(z.re)) / T(2));
  if (z.re >= T(0)) return {a, z.im / (T(2) * a)};
  T b = z.im / (T(2) * a);
  return (z.im >= T(0)) ? Cx<T>{tabs(b), a} : Cx<T>{tabs(b), -a};
}
template <class T> Cx<T> cdiv(Cx<T> a, Cx<T> b) {
  T den = b.re * b.re + b.im * b.im;
  return {(a.re * b.re + a.im * b.im) / den, (a.im * b.re - a.re * b.im) / den};
}

template <class T> std::vector<Cx<T>> load(const double* A, int n) {
  std::vector<Cx<T>> M((size_t)n * n);
  for (size_t i = 0; i < (size_t)n * n; ++i) M[i] = {T(A[2 * i]), T(A[2 * i + 1])};
  return M;
}

// Split a value of type T into (hi, lo) binary64 words.
inline void put(double x, double* o) { o[0] = x; o[1] = 0.0; }
inline void put(__float128 x, double* o) {
  double hi = (double)x;
  o[0] = hi;
  o[1] = (double)(x - (__float128)hi);
}
template <class T> void put_c(Cx<T> z, double* o) { put(z.re, o); put(z.im, o + 2); }

// ---------------------------------------------------------------- permanent
// Glynn: perm(A) = 2^-(n-1) sum_delta (prod delta) prod_r (sum_c delta_c A[r,c]),
// delta_0 = +1, Gray order over delta_1..delta_{n-1}; cpu_ref/permanent.py:108-139.
template <class T> Cx<T> perm_glynn(const std::vector<Cx<T>>& M, int n, double* absnorm) {
  if (n == 0) { if (absnorm) *absnorm = 1.0; return {T(1), T(0)}; }
  std::vector<Cx<T>> rowsum(n);
  for (int r = 0; r < n; ++r) {
    Cx<T> s{T(0), T(0)};
    for (int c = 0; c < n; ++c) s = cadd(s, M[(size_t)r * n + c]);
    rowsum[r] = s;
  }
  auto prod = [&]() {
    Cx<T> p = rowsum[0];
    for (int r = 1; r < n; ++r) p = cmul(p, rowsum[r]);
    return p;
  };
  Cx<T> p0 = prod();
  Cx<T> total = p0;
  double abs_acc = cabs_d(p0);
  int sign = 1;
  const uint64_t terms = 1ull << (n - 1);
  for (uint64_t i = 1; i < terms; ++i) {
    int k = __builtin_ctzll(i);
    int col = k + 1;
    T step = (((i ^ (i >> 1)) >> k) & 1ull) ? T(-2) : T(2);
    for (int r = 0; r < n; ++r) rowsum[r] = cadd(rowsum[r], cscale(M[(size_t)r * n + col], step));
    sign = -sign;
    Cx<T> p = prod();
    total = sign > 0 ? cadd(total, p) : csub(total, p);
    abs_acc += cabs_d(p);
  }
  if (absnorm) *absnorm = abs_acc / (double)terms;
  return cscale(total, T(1) / T((double)terms));
}

// ---------------------------------------------------------------- hafnians
// [lambda^n] exp(sum_k g_k lambda^k) from kg[k] = k g_k: e_j = (1/j) sum_k kg[k] e_{j-k};
// cpu_ref/hafnian.py:62-80.
template <class T> Cx<T> exp_coeff_from_kg(const std::vector<Cx<T>>& kg, int n) {
  std::vector<Cx<T>> e(n + 1);
  e[0] = {T(1), T(0)};
  for (int j = 1; j <= n; ++j) {
    Cx<T> acc{T(0), T(0)};
    for (int k = 1; k <= j; ++k) acc = cadd(acc, cmul(kg[k], e[j - k]));
    e[j] = {acc.re / T(j), acc.im / T(j)};
  }
  return e[n];
}

// One subset term of the (loop) hafnian: (-1)^(n-m) [lambda^n] exp(...) for C = B_S X.
// loop=false: ordinary hafnian, diagonal zeroed (cpu_ref/hafnian.py:116).
// loop=true: kg[k] = p_k/2 + k * (1/2) d^T X C^{k-1} d (cpu_ref/loop_hafnian.py:94-104).
template <class T>
Cx<T> haf_subset_term(const std::vector<Cx<T>>& M, int N, int n, uint64_t mask, bool loop) {
  int m = __builtin_popcountll(mask);
  std::vector<Cx<T>> kg(n + 1, Cx<T>{T(0), T(0)});
  if (m == 0) {
    // [lambda^n] exp(0) = [n == 0]; n >= 1 here.
    return {T(0), T(0)};
  }
  int s = 2 * m;
  std::vector<int> idx;
  for (int i = 0; i < n; ++i)
    if ((mask >> i) & 1ull) { idx.push_back(2 * i); idx.push_back(2 * i + 1); }
  std::vector<Cx<T>> C((size_t)s * s), d(s);
  for (int r = 0; r < s; ++r) {
    for (int c = 0; c < s; ++c) {
      int cc = idx[c ^ 1];  // B X: swap columns within each pair
      Cx<T> v = M[(size_t)idx[r] * N + cc];
      if (!loop && idx[r] == cc) v = {T(0), T(0)};  // ordinary hafnian: zero diagonal
      C[(size_t)r * s + c] = v;
    }
    d[r] = M[(size_t)idx[r] * N + idx[r]];
  }
  // power traces p_k = tr(C^k), k = 1..n, by P <- P C (cpu_ref/hafnian.py:83-93)
  std::vector<Cx<T>> P = C, Q((size_t)s * s), Tm((size_t)s * s);
  // Q = C^{k-1} for the loop term, starting from the identity
  for (int i = 0; i < s * s; ++i) Q[i] = {T(0), T(0)};
  for (int i = 0; i < s; ++i) Q[(size_t)i * s + i] = {T(1), T(0)};
  for (int k = 1; k <= n; ++k) {
    Cx<T> pk{T(0), T(0)};
    for (int i = 0; i < s; ++i) pk = cadd(pk, P[(size_t)i * s + i]);
    Cx<T> half_pk = cscale(pk, T(0.5));
    if (loop) {
      // v_k = 1/2 d^T X Q d ; X swaps entries within each pair
      Cx<T> vk{T(0), T(0)};
      for (int a = 0; a < s; ++a) {
        Cx<T> w{T(0), T(0)};
        for (int c = 0; c < s; ++c) w = cadd(w, cmul(Q[(size_t)(a ^ 1) * s + c], d[c]));
        vk = cadd(vk, cmul(d[a], w));
      }
      vk = cscale(vk, T(0.5));
      kg[k] = cadd(half_pk, cscale(vk, T(k)));
    } else {
      kg[k] = half_pk;
    }
    if (k < n) {
      if (loop) Q = P;
      for (int i = 0; i < s; ++i)
        for (int j = 0; j < s; ++j) {
          Cx<T> acc{T(0), T(0)};
          for (int t = 0; t < s; ++t) acc = cadd(acc, cmul(P[(size_t)i * s + t], C[(size_t)t * s + j]));
          Tm[(size_t)i * s + j] = acc;
        }
      P.swap(Tm);
    }
  }
  Cx<T> coeff = exp_coeff_from_kg(kg, n);
  return ((n - m) & 1) ? Cx<T>{-coeff.re, -coeff.im} : coeff;
}

template <class T> Cx<T> haf_powertrace(std::vector<Cx<T>> M, int N, bool loop, double* absnorm) {
  if (N == 0) { if (absnorm) *absnorm = 1.0; return {T(1), T(0)}; }
  if (N & 1) {
    if (!loop) { if (absnorm) *absnorm = 0.0; return {T(0), T(0)}; }
    // lhaf(A_odd) = lhaf(A_odd (+) [1])  (gbskernels/__init__.py:190-200)
    std::vector<Cx<T>> aug((size_t)(N + 1) * (N + 1), Cx<T>{T(0), T(0)});
    for (int r = 0; r < N; ++r)
      for (int c = 0; c < N; ++c) aug[(size_t)r * (N + 1) + c] = M[(size_t)r * N + c];
    aug[(size_t)N * (N + 1) + N] = {T(1), T(0)};
    M.swap(aug);
    N += 1;
  }
  int n = N / 2;
  Cx<T> total{T(0), T(0)};
  double abs_acc = 0.0;
  for (uint64_t mask = 0; mask < (1ull << n); ++mask) {
    Cx<T> t = haf_subset_term(M, N, n, mask, loop);
    total = cadd(total, t);
    abs_acc += cabs_d(t);
  }
  if (absnorm) *absnorm = abs_acc;
  return total;
}

// ---------------------------------------------------------------- torontonians
// Real recursive prefix Cholesky over the mode lattice, xxpp ordering, DFS with
// exclude-first order: core/tor_recursive.cu:41-115.  Returns NaN if a leading
// minor of I - O_S is not positive definite (off the physical domain).
template <class T> struct TorRec {
  const std::vector<T>& O;
  int n, dim;
  std::vector<T> L;
  std::vector<int> modes;
  T total{0};
  double abs_acc = 0.0;
  bool bad = false;
  TorRec(const std::vector<T>& O_, int n_) : O(O_), n(n_), dim(2 * n_), L((size_t)4 * n_ * n_), modes(n_) {}

  bool append(int j, int count, T& dprod) {
    int size = 2 * count;
    modes[count] = j;
    for (int t = 0; t < 2; ++t) {
      int r = size + t;
      int gj = t == 0 ? j : j + n;
      for (int c = 0; c <= r; ++c) {
        int mc = ((c >> 1) == count) ? j : modes[c >> 1];
        int gc = (c & 1) ? mc + n : mc;
        T s = ((gj == gc) ? T(1) : T(0)) - O[(size_t)gj * dim + gc];
        for (int u = 0; u < c; ++u) s -= L[(size_t)r * dim + u] * L[(size_t)c * dim + u];
        if (c < r) {
          L[(size_t)r * dim + c] = s / L[(size_t)c * dim + c];
        } else {
          if (!(s > T(0))) return false;
          L[(size_t)r * dim + r] = tsqrt(s);
        }
      }
    }
    T a = L[(size_t)size * dim + size], b = L[(size_t)(size + 1) * dim + size + 1];
    dprod = (a * b) * (a * b);
    return true;
  }
  void rec(int mode, int count, T detprod) {
    if (bad) return;
    if (mode == n) {
      T c = T(1) / tsqrt(detprod);
      total += ((n - count) & 1) ? -c : c;
      abs_acc += to_d(c);
      return;
    }
    rec(mode + 1, count, detprod);
    T d;
    if (!append(mode, count, d)) { bad = true; return; }
    rec(mode + 1, count + 1, detprod * d);
  }
};

// Per-subset determinant torontonian with complex LU + partial pivoting and the
// principal square root: cpu_ref/torontonian.py:48-64 (np.linalg.det + np.sqrt).
template <class T> Cx<T> det_lu(std::vector<Cx<T>>& a, int s) {
  Cx<T> det{T(1), T(0)};
  for (int k = 0; k < s; ++k) {
    int piv = k;
    T best = cabs_t(a[(size_t)k * s + k]);
    for (int i = k + 1; i < s; ++i) {
      T v = cabs_t(a[(size_t)i * s + k]);
      if (v > best) { best = v; piv = i; }
    }
    if (best == T(0)) return {T(0), T(0)};
    if (piv != k) {
      for (int j = 0; j < s; ++j) std::swap(a[(size_t)k * s + j], a[(size_t)piv * s + j]);
      det = {-det.re, -det.im};
    }
    Cx<T> p = a[(size_t)k * s + k];
    det = cmul(det, p);
    for (int i = k + 1; i < s; ++i) {
      Cx<T> f = cdiv(a[(size_t)i * s + k], p);
      for (int j = k + 1; j < s; ++j) a[(size_t)i * s + j] = csub(a[(size_t)i * s + j], cmul(f, a[(size_t)k * s + j]));
    }
  }
  return det;
}

template <class T> Cx<T> tor_subset_det(const std::vector<Cx<T>>& M, int n, double* absnorm) {
  int dim = 2 * n;
  Cx<T> total{T(0), T(0)};
  double abs_acc = 0.0;
  for (uint64_t mask = 0; mask < (1ull << n); ++mask) {
    std::vector<int> idx;
    for (int i = 0; i < n; ++i) if ((mask >> i) & 1ull) idx.push_back(i);
    int m = (int)idx.size();
    for (int i = 0; i < m; ++i) idx.push_back(idx[i] + n);
    int s = 2 * m;
    std::vector<Cx<T>> a((size_t)s * s);
    for (int r = 0; r < s; ++r)
      for (int c = 0; c < s; ++c) {
        Cx<T> v = M[(size_t)idx[r] * dim + idx[c]];
        a[(size_t)r * s + c] = {((r == c) ? T(1) : T(0)) - v.re, -v.im};
      }
    Cx<T> det = s ? det_lu(a, s) : Cx<T>{T(1), T(0)};
    Cx<T> term = cdiv(Cx<T>{T(1), T(0)}, csqrt_principal(det));
    if ((n - m) & 1) term = {-term.re, -term.im};
    total = cadd(total, term);
    abs_acc += cabs_d(term);
  }
  if (absnorm) *absnorm = abs_acc;
  return total;
}

template <class T> void tor_real(const double* O, int n, double* out, double* absnorm) {
  if (n == 0) { put(T(1), out); out[2] = out[3] = 0.0; if (absnorm) *absnorm = 1.0; return; }
  std::vector<T> OT((size_t)4 * n * n);
  for (size_t i = 0; i < OT.size(); ++i) OT[i] = T(O[i]);
  TorRec<T> tr(OT, n);
  tr.rec(0, 0, T(1));
  if (tr.bad) {
    out[0] = out[1] = NAN; out[2] = out[3] = 0.0;
    if (absnorm) *absnorm = NAN;
    return;
  }
  put(tr.total, out);
  out[2] = out[3] = 0.0;
  if (absnorm) *absnorm = tr.abs_acc;
}

// Loop hafnian of A (M x M) with row / column i repeated reps[i] times and loop
// weight gamma[i] on every copy: the finite-difference sieve of
// cpu_ref/repeated.py:64-122 (same enumeration order: all v <= reps in row-major
// odometer order, the v <-> reps - v symmetry keeping v lexicographically <= its
// mirror and doubling the strict half; S_N by the mu-power ladder and the running
// sigma^2 power, as there).
template <class T> Cx<T> lhaf_sieve(const double* A, const double* g, const int* reps, int M) {
  int N = 0;
  for (int i = 0; i < M; ++i) N += reps[i];
  if (N == 0) return {T(1), T(0)};
  const int kmax = N / 2;
  std::vector<T> coeff(kmax + 1);
  for (int k = 0; k <= kmax; ++k) {
    // C(N, 2k) (2k-1)!! accumulated in T
    T c = T(1);
    for (int t = 1; t <= 2 * k; ++t) c = c * T(N - 2 * k + t) / T(t);
    for (int t = 2 * k - 1; t > 0; t -= 2) c = c * T(t);
    coeff[k] = c;
  }
  auto binom = [](int n, int k) {
    T c = T(1);
    for (int t = 1; t <= k; ++t) c = c * T(n - k + t) / T(t);
    return c;
  };
  std::vector<int> v(M, 0);
  std::vector<T> x(M);
  Cx<T> total{T(0), T(0)};
  for (;;) {
    // lexicographic comparison of v with its mirror reps - v
    int cmp = 0;
    for (int i = 0; i < M && cmp == 0; ++i) {
      const int mi = reps[i] - v[i];
      cmp = v[i] < mi ? -1 : (v[i] > mi ? 1 : 0);
    }
    if (cmp <= 0) {
      int vs = 0;
      for (int i = 0; i < M; ++i) vs += v[i];
      T c = (vs % 2 == 0) ? T(1) : T(-1);
      if (cmp < 0) c = c * T(2);
      for (int i = 0; i < M; ++i) c = c * binom(reps[i], v[i]);
      for (int i = 0; i < M; ++i) x[i] = T(reps[i] - 2 * v[i]);
      Cx<T> sig2{T(0), T(0)}, mu{T(0), T(0)};
      for (int i = 0; i < M; ++i) {
        Cx<T> row{T(0), T(0)};
        for (int j = 0; j < M; ++j)
          row = cadd(row, cscale(Cx<T>{T(A[2 * (i * M + j)]), T(A[2 * (i * M + j) + 1])}, x[j]));
        sig2 = cadd(sig2, cscale(row, x[i]));
        mu = cadd(mu, cscale(Cx<T>{T(g[2 * i]), T(g[2 * i + 1])}, x[i]));
      }
      std::vector<Cx<T>> mupow(kmax + 1);
      mupow[kmax] = (N % 2) ? mu : Cx<T>{T(1), T(0)};
      const Cx<T> mu2 = cmul(mu, mu);
      for (int k = kmax - 1; k >= 0; --k) mupow[k] = cmul(mupow[k + 1], mu2);
      Cx<T> SN{T(0), T(0)}, sk{T(1), T(0)};
      for (int k = 0; k <= kmax; ++k) {
        SN = cadd(SN, cmul(cscale(sk, coeff[k]), mupow[k]));
        sk = cmul(sk, sig2);
      }
      total = cadd(total, cscale(SN, c));
    }
    int i = M - 1;  // odometer, last index fastest (numpy ndindex order)
    while (i >= 0 && v[i] == reps[i]) v[i--] = 0;
    if (i < 0) break;
    ++v[i];
  }
  T D = T(1);
  for (int t = 2; t <= N; ++t) D = D * T(t);
  for (int t = 0; t < N; ++t) D = D * T(2);
  return cscale(total, T(1) / D);
}

}  // namespace

extern "C" {

// prec: 0 = binary64, 1 = binary128.  out: 4 doubles (re_hi, re_lo, im_hi, im_lo).
// absnorm (may be null): sum|term| in the reference's normalisation.
int orc_perm(const double* A, int n, int prec, double* out, double* absnorm) {
  if (n < 0 || n > 40) return 1;
  if (prec == 0) put_c(perm_glynn<double>(load<double>(A, n), n, absnorm), out);
  else put_c(perm_glynn<__float128>(load<__float128>(A, n), n, absnorm), out);
  return 0;
}

int orc_haf(const double* A, int N, int prec, double* out, double* absnorm) {
  if (N < 0 || N > 64) return 1;
  if (prec == 0) put_c(haf_powertrace<double>(load<double>(A, N), N, false, absnorm), out);
  else put_c(haf_powertrace<__float128>(load<__float128>(A, N), N, false, absnorm), out);
  return 0;
}

int orc_lhaf(const double* A, int N, int prec, double* out, double* absnorm) {
  if (N < 0 || N > 64) return 1;
  if (prec == 0) put_c(haf_powertrace<double>(load<double>(A, N), N, true, absnorm), out);
  else put_c(haf_powertrace<__float128>(load<__float128>(A, N), N, true, absnorm), out);
  return 0;
}

// Real O (2n x 2n binary64, row-major), recursive prefix Cholesky. NaN = off-domain.
int orc_tor_real(const double* O, int n, int prec, double* out, double* absnorm) {
  if (n < 0 || n > 40) return 1;
  if (prec == 0) tor_real<double>(O, n, out, absnorm);
  else tor_real<__float128>(O, n, out, absnorm);
  return 0;
}

// Complex O (2n x 2n complex128), per-subset LU determinant.
int orc_tor_complex(const double* O, int n, int prec, double* out, double* absnorm) {
  if (n < 0 || n > 30) return 1;
  if (n == 0) { out[0] = 1.0; out[1] = out[2] = out[3] = 0.0; if (absnorm) *absnorm = 1.0; return 0; }
  if (prec == 0) put_c(tor_subset_det<double>(load<double>(O, 2 * n), n, absnorm), out);
  else put_c(tor_subset_det<__float128>(load<__float128>(O, 2 * n), n, absnorm), out);
  return 0;
}

// Repeated-row loop hafnian (finite-difference sieve): A (M x M complex), gamma (M
// complex, may be null = 0), reps (M ints).
int orc_lhaf_repeated(const double* A, const double* gamma, const int* reps, int M, int prec, double* out) {
  if (M < 0 || M > 64) return 1;
  std::vector<double> g0;
  if (!gamma) {
    g0.assign(2 * (size_t)std::max(M, 1), 0.0);
    gamma = g0.data();
  }
  for (int i = 0; i < M; ++i)
    if (reps[i] < 0) return 1;
  if (prec == 0) put_c(lhaf_sieve<double>(A, gamma, reps, M), out);
  else put_c(lhaf_sieve<__float128>(A, gamma, reps, M), out);
  return 0;
}

}  // extern "C"
