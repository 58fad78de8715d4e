// gbs_items.cuh -- the work-item kernel behind every batched evaluation.
//
// One kernel template serves the plain per-size launches (a single (function,
// tier) branch compiled in, lean registers) and the persistent mixed-size queue
// (several branches compiled in): warps pull work items from a device queue head
// with one atomic each, evaluate, publish a partial, and the warp that finishes
// the last item of an instance reduces that instance's partials in item order.
// No warp ever waits on another, so there is no spin anywhere in the kernel.
#pragma once
#include <cuda_runtime.h>

#include <atomic>
#include <mutex>

#include "gbs_common.cuh"
#include "gbs_kernels.cuh"
#include "haf_dd.cuh"
#include "haf_pt.cuh"
#include "perm_tor.cuh"
#include "cert.cuh"
#include "tor_lu.cuh"
#include "tor_warp.cuh"
#include "tor_warp_dd.cuh"

namespace gbsb {


// ------------------------------------------------------------------ item evaluators
struct ItemResult {
  ddc val;
  double aux;
  int st;
};

__device__ __forceinline__ ddc ddc_from_c(cplx v) { return ddc{dd_make(v.re), dd_make(v.im)}; }

// Permanent item: Gray indices [lo, lo + count), 32 lanes x R = count / 32 each
// (count < 32 only when the whole walk is shorter than a warp).
template <int NN, int TIER>
__device__ ItemResult perm_item_n(const double* A2, unsigned long long lo, unsigned long long count, int lane) {
  ItemResult r{ddc{dd_make(0.0), dd_make(0.0)}, 0.0, kStOk};
  unsigned long long R = count >= 32 ? count / 32 : 1;
  bool active = count >= 32 || (unsigned long long)lane < count;
  unsigned long long i0 = lo + (unsigned long long)lane * R;
  if (TIER == kTierDD) {
    ddc v = ddc{dd_make(0.0), dd_make(0.0)};
    if (active) v = perm_lane_range_dd<NN>(A2, i0, R);
    r.val = warp_sum_ddc(v);
  } else if (TIER == kTierCert) {
    cball b{mkc(0.0, 0.0), 0.0};
    if (active) b = perm_lane_range_cert<NN>(A2, i0, R);
    b = warp_sum_cb(b);
    r.val = ddc_from_c(b.z);
    r.aux = b.r;
  } else if (TIER == kTierCertDD) {
    ddball b{ddc{dd_make(0.0), dd_make(0.0)}, 0.0};
    if (active) b = perm_lane_range_certdd<NN>(A2, i0, R);
    b = warp_sum_ddb(b);
    r.val = b.z;
    r.aux = b.r;
  } else {
    double absacc = 0.0;
    cplx v = mkc(0.0, 0.0);
    if (active) v = perm_lane_range<NN, TIER == kTierKappa>(A2, i0, R, absacc);
    v = warp_sum_c(v);
    r.val = ddc_from_c(v);
    if (TIER == kTierKappa) r.aux = warp_sum_d(absacc);
  }
  return r;
}

template <int TIER>
__device__ ItemResult perm_item(const double* __restrict__ mats, const InstDesc& d, const WorkItem& w,
                                double* ws, int lane) {
  const int n = d.dim;
  const double* A = mats + d.off;
  // stage 2A (exact scaling) in this warp's shared workspace
  for (int e = lane; e < n * n; e += 32) st_c(ws + e * 2, cscale(ld_c(A + e * 2), 2.0));
  __syncwarp();
  ItemResult r;
  switch (n) {
#define GBSB_PERM_CASE(K) \
  case K: r = perm_item_n<K, TIER>(ws, w.lo, w.count, lane); break;
    GBSB_PERM_CASE(1) GBSB_PERM_CASE(2) GBSB_PERM_CASE(3) GBSB_PERM_CASE(4) GBSB_PERM_CASE(5)
    GBSB_PERM_CASE(6) GBSB_PERM_CASE(7) GBSB_PERM_CASE(8) GBSB_PERM_CASE(9) GBSB_PERM_CASE(10)
    GBSB_PERM_CASE(11) GBSB_PERM_CASE(12) GBSB_PERM_CASE(13) GBSB_PERM_CASE(14) GBSB_PERM_CASE(15)
    GBSB_PERM_CASE(16) GBSB_PERM_CASE(17) GBSB_PERM_CASE(18) GBSB_PERM_CASE(19) GBSB_PERM_CASE(20)
    GBSB_PERM_CASE(21) GBSB_PERM_CASE(22) GBSB_PERM_CASE(23) GBSB_PERM_CASE(24) GBSB_PERM_CASE(25)
    GBSB_PERM_CASE(26) GBSB_PERM_CASE(27) GBSB_PERM_CASE(28)
#undef GBSB_PERM_CASE
    default:
      r = ItemResult{ddc{dd_make(0.0), dd_make(0.0)}, 0.0, kStTooLarge};
  }
  __syncwarp();
  return r;
}

// REAL: the instance is real (binary64 tiers; the host sets InstDesc::real_in) and
// runs the real power loop.  A separate instantiation, so the complex code is
// compiled as if the real path did not exist.
template <int TIER, bool REAL = false>
__device__ __noinline__ ItemResult haf_item(const double* __restrict__ mats, const InstDesc& d, const WorkItem& w,
                               bool loop, double* ws, int haf_smax, int lane) {
  ItemResult r{ddc{dd_make(0.0), dd_make(0.0)}, 0.0, kStOk};
  const int N = d.dim, n = N / 2;
  const double* A = mats + d.off;
  if (TIER == kTierDD) {
    const HafDDLayout L = haf_dd_layout(haf_smax);
    ddc acc = ddc{dd_make(0.0), dd_make(0.0)};
    for (unsigned long long k = 0; k < w.count; ++k) {
      ddc t = haf_subset_term_dd<false>(A, N, n, (uint32_t)(w.lo + k), loop, ws, L, lane).z;
      acc = ddc_add(acc, t);
    }
    r.val = acc;
  } else if (TIER == kTierCertDD) {
    // the dd walk and its subset sum, as balls (the value is the dd value bit for bit)
    const HafDDLayout L = haf_dd_layout(haf_smax, true);
    ddball acc{ddc{dd_make(0.0), dd_make(0.0)}, 0.0};
    for (unsigned long long k = 0; k < w.count; ++k) {
      const ddball t = haf_subset_term_dd<true>(A, N, n, (uint32_t)(w.lo + k), loop, ws, L, lane);
      acc = ddb_add(acc, t);
    }
    r.val = acc.z;
    r.aux = acc.r;
    if (!isfinite(acc.r) || !isfinite(acc.z.re.hi) || !isfinite(acc.z.im.hi)) r.st = kStUncertified;
  } else if (TIER == kTierCert) {
    // same grouping as the binary64 tiers (rings of kHafRing subsets, butterfly sum
    // per ring) so the certified value is the fp64 value bit for bit
    const HafLayout L = haf_layout(haf_smax, true);
    double* ring = ws + L.cring_off;
    cball acc{mkc(0.0, 0.0), 0.0};
    int cnt = 0;
    for (unsigned long long k = 0; k < w.count; ++k) {
      // each subset parks its kg balls; kHafRing lanes then run the recurrences at once
      haf_subset_term_tc<true, REAL>(A, N, n, (uint32_t)(w.lo + k), loop, ws, L, lane, ring + cnt * L.cslot);
      if (++cnt == kHafRing || k + 1 == w.count) {
        __syncwarp();
        acc = cb_add(acc, haf_ring_flush_cert(ring, L.cslot, cnt, n, lane, ws + L.p_off));
        cnt = 0;
        __syncwarp();
      }
    }
    r.val = ddc_from_c(acc.z);
    r.aux = acc.r;
    if (!isfinite(acc.r) || !isfinite(acc.z.re) || !isfinite(acc.z.im)) r.st = kStUncertified;
  } else {
    // the traces of kHafRing subsets are parked, then kHafRing lanes run their
    // Newton recurrences at once (see haf_ring_flush)
    const HafLayout L = haf_layout(haf_smax);
    double* ring = ws + L.ring_off;
    cplx acc = mkc(0.0, 0.0);
    double absacc = 0.0;
    int cnt = 0;
    for (unsigned long long k = 0; k < w.count; ++k) {
      haf_subset_term_tc<false, REAL>(A, N, n, (uint32_t)(w.lo + k), loop, ws, L, lane, ring + cnt * L.slot * 2);
      if (++cnt == kHafRing || k + 1 == w.count) {
        __syncwarp();
        double ab = 0.0;
        const cplx t = haf_ring_flush(ring, L.slot, cnt, n, lane, TIER == kTierKappa ? &ab : nullptr,
                                      ws + L.p_off);
        acc = cadd(acc, t);
        absacc += ab;
        cnt = 0;
        __syncwarp();
      }
    }
    r.val = ddc_from_c(acc);
    r.aux = absacc;
  }
  return r;
}

template <int TIER>
__device__ ItemResult tor_item(const double* __restrict__ mats, const InstDesc& d, const WorkItem& w,
                               double* ws, int lane) {
  ItemResult r{ddc{dd_make(0.0), dd_make(0.0)}, 0.0, kStOk};
  const int n = d.dim / 2;
  const int dim = d.dim;
  const double* Oc = mats + d.off;
  if (!d.real_in) {
    // complex O (binary64 tiers only; the host refuses the others): one warp per
    // subset LU, w.count masks from w.lo (tor_lu.cuh); the certified tier carries
    // ball radii through the same LU (value = the fp64 value bit for bit)
    if constexpr (TIER == kTierFp64 || TIER == kTierKappa || TIER == kTierCert) {
      constexpr bool CERT = TIER == kTierCert;
      cball acc{mkc(0.0, 0.0), 0.0};
      double aabs = 0.0;
      bool sing = false;
      for (unsigned long long k = 0; k < w.count; ++k) {
        const cball t = tor_lu_term<CERT>(Oc, n, (uint32_t)(w.lo + k), ws, lane, sing);
        if constexpr (CERT) acc = cb_add(acc, t);
        else acc.z = cadd(acc.z, t.z);
        if (TIER == kTierKappa) aabs += hypot(t.z.re, t.z.im);
        __syncwarp();
      }
      r.val = ddc_from_c(acc.z);
      r.aux = CERT ? acc.r : aabs;
      if (sing) r.st = CERT ? kStUncertified : kStOffDomain;
      else if (CERT && !(acc.r < INFINITY)) r.st = kStUncertified;
    } else {
      r.st = kStTooLarge;
    }
    return r;
  }
  if constexpr (TIER != kTierDD && TIER != kTierCertDD) {
    // binary64 tiers: warp-cooperative prefix walk with the 32-subset register tail
    // (tor_warp.cuh); one work item = w.count prefix patterns over the first d.param
    // prefix modes, walked one after another by the whole warp
    const TorWLayout Lw = tor_w_layout(n, TIER == kTierCert);
    double* rho = ws + Lw.rho_off;
    bool proved = true;
    if (TIER == kTierCert) {
      double dmin2 = 0.0;
      const double sigma = tor_cert_sigma(Oc, n, ws + Lw.col_off, lane, dmin2);
      proved = sigma > 0.0;
      tor_cert_rho(sigma, dmin2, n, rho, lane);
    }
    double val = 0.0, aux = 0.0;
    bool ok = true;
    if (proved) {
      for (unsigned long long p = 0; p < w.count; ++p) {
        double t = 0.0, a = 0.0;
        ok = tor_warp_item<TIER == kTierKappa, TIER == kTierCert>(Oc, n, d.param, (uint32_t)(w.lo + p), ws, Lw,
                                                                   rho, lane, t, a) && ok;
        if (p == 0) {
          val = t;
          aux = a;
        } else if (TIER == kTierCert) {
          val += t;
          aux = ru_add(ru_add(aux, a), ru_mul(kUc, fabs(val)));
        } else {
          val += t;
          aux += a;
        }
      }
    }
    r.val = ddc{dd_make(val), dd_make(0.0)};
    r.aux = aux;
    if (!proved || !ok) r.st = TIER == kTierCert ? kStUncertified : kStOffDomain;
    __syncwarp();
    return r;
  } else {
    // double-double tiers: the same walk in double-word arithmetic with a 16-subset
    // tail (tor_warp_dd.cuh); one work item = w.count prefix patterns.  The certified
    // tier adds the radius (same value bit for bit).
    constexpr bool CERT = TIER == kTierCertDD;
    const TorDLayout Lw = tor_d_layout(n, CERT);
    double* rho = ws + Lw.rho_off;
    bool proved = true;
    if (CERT) {
      double dmin2 = 0.0;
      const double sigma = tor_cert_sigma(Oc, n, ws + Lw.col_off, lane, dmin2);
      proved = sigma > 0.0;
      tor_cert_rho_dd(sigma, dmin2, n, rho, lane);
    }
    dd val = dd_make(0.0);
    double aux = 0.0;
    bool ok = true;
    if (proved) {
      for (unsigned long long p = 0; p < w.count; ++p) {
        dd t = dd_make(0.0);
        double a = 0.0;
        ok = tor_dd_item<CERT>(Oc, n, d.param, (uint32_t)(w.lo + p), ws, Lw, rho, lane, t, a) && ok;
        if (p == 0) {
          val = t;
          aux = a;
        } else {
          val = dd_add(val, t);
          if (CERT) aux = ru_add(ru_add(aux, a), ru_add(ru_mul(4.0 * kU * kU, fabs(val.hi)), kUfl));
        }
      }
    }
    r.val = ddc{val, dd_make(0.0)};
    r.aux = aux;
    if (!proved || !ok) r.st = CERT ? kStUncertified : kStOffDomain;
    __syncwarp();
    return r;
  }
}

// ------------------------------------------------------------------ the item kernel
template <unsigned BR>
__device__ __forceinline__ ItemResult eval_item(const ItemLaunch& P, const InstDesc& d, const WorkItem& w,
                                                double* ws, int lane) {
  ItemResult r{ddc{dd_make(0.0), dd_make(0.0)}, 0.0, kStTooLarge};
  switch (d.ft) {
// binary64 hafnian tiers: the real instantiation for a real instance
#define GBSB_HAF(TIER, LOOP)                                                     \
  (d.real_in ? haf_item<TIER, true>(P.mats, d, w, LOOP, ws, P.haf_smax, lane)   \
             : haf_item<TIER, false>(P.mats, d, w, LOOP, ws, P.haf_smax, lane))
#define GBSB_BR(FN, TIER, CALL) \
  case ft_code(FN, TIER):         \
    if constexpr ((BR >> ft_code(FN, TIER)) & 1u) { r = CALL; } \
    break;
    GBSB_BR(kFnPerm, kTierFp64, (perm_item<kTierFp64>(P.mats, d, w, ws, lane)))
    GBSB_BR(kFnPerm, kTierKappa, (perm_item<kTierKappa>(P.mats, d, w, ws, lane)))
    GBSB_BR(kFnPerm, kTierDD, (perm_item<kTierDD>(P.mats, d, w, ws, lane)))
    GBSB_BR(kFnHaf, kTierFp64, (GBSB_HAF(kTierFp64, false)))
    GBSB_BR(kFnHaf, kTierKappa, (GBSB_HAF(kTierKappa, false)))
    GBSB_BR(kFnHaf, kTierDD, (haf_item<kTierDD>(P.mats, d, w, false, ws, P.haf_smax, lane)))
    GBSB_BR(kFnLhaf, kTierFp64, (GBSB_HAF(kTierFp64, true)))
    GBSB_BR(kFnLhaf, kTierKappa, (GBSB_HAF(kTierKappa, true)))
    GBSB_BR(kFnLhaf, kTierDD, (haf_item<kTierDD>(P.mats, d, w, true, ws, P.haf_smax, lane)))
    GBSB_BR(kFnTor, kTierFp64, (tor_item<kTierFp64>(P.mats, d, w, ws, lane)))
    GBSB_BR(kFnTor, kTierKappa, (tor_item<kTierKappa>(P.mats, d, w, ws, lane)))
    GBSB_BR(kFnTor, kTierDD, (tor_item<kTierDD>(P.mats, d, w, ws, lane)))
    GBSB_BR(kFnPerm, kTierCert, (perm_item<kTierCert>(P.mats, d, w, ws, lane)))
    GBSB_BR(kFnPerm, kTierCertDD, (perm_item<kTierCertDD>(P.mats, d, w, ws, lane)))
    GBSB_BR(kFnHaf, kTierCert, (GBSB_HAF(kTierCert, false)))
    GBSB_BR(kFnLhaf, kTierCert, (GBSB_HAF(kTierCert, true)))
    GBSB_BR(kFnHaf, kTierCertDD, (haf_item<kTierCertDD>(P.mats, d, w, false, ws, P.haf_smax, lane)))
    GBSB_BR(kFnLhaf, kTierCertDD, (haf_item<kTierCertDD>(P.mats, d, w, true, ws, P.haf_smax, lane)))
    GBSB_BR(kFnTor, kTierCert, (tor_item<kTierCert>(P.mats, d, w, ws, lane)))
    GBSB_BR(kFnTor, kTierCertDD, (tor_item<kTierCertDD>(P.mats, d, w, ws, lane)))
#undef GBSB_BR
#undef GBSB_HAF
    default:
      break;
  }
  return r;
}

template <unsigned BR>
__global__ void __launch_bounds__(256) gbs_items_kernel(ItemLaunch P) {
  extern __shared__ __align__(128) double smem[];
  const int lane = threadIdx.x & 31;
  const int warp = threadIdx.x >> 5;
  double* ws = smem + (size_t)warp * P.ws_doubles;
  const int n_items = P.n_items_dev ? *P.n_items_dev : P.n_items;
  for (;;) {
    int it = 0;
    if (lane == 0) it = atomicAdd(P.head, 1);
    it = __shfl_sync(0xffffffffu, it, 0);
    if (it >= n_items) break;
    if (P.order) it = P.order[it];
    const WorkItem w = P.items[it];
    const InstDesc d = P.insts[w.inst];
    ItemResult r = eval_item<BR>(P, d, w, ws, lane);
    int last = 0;
    if (lane == 0) {
      double4 pv = make_double4(r.val.re.hi, r.val.re.lo, r.val.im.hi, r.val.im.lo);
      *reinterpret_cast<double4*>(P.part + (size_t)it * 4) = pv;
      P.paux[it] = r.aux;
      P.pst[it] = r.st;
      __threadfence();
      const int old = atomicAdd(P.done + w.inst, 1);
      last = (old == d.nitems - 1);
    }
    last = __shfl_sync(0xffffffffu, last, 0);
    if (last) {
      __threadfence();
      // Deterministic reduction: lane l sums items l, l+32, ... in order, then a
      // fixed butterfly combines the lanes.  Partials are read through L2.
      const bool cert = tier_certified(ft_tier(d.ft));
      ddc acc = ddc{dd_make(0.0), dd_make(0.0)};
      double aux = 0.0, mag = 0.0;
      int st = kStOk;
      for (int k = lane; k < d.nitems; k += 32) {
        const double* pp = P.part + (size_t)(d.item0 + k) * 4;
        ddc v = ddc{dd{__ldcg(pp), __ldcg(pp + 1)}, dd{__ldcg(pp + 2), __ldcg(pp + 3)}};
        acc = ddc_add(acc, v);
        const double a = __ldcg(P.paux + d.item0 + k);
        aux = cert ? ru_add(aux, a) : aux + a;
        if (cert) mag = ru_add(mag, ru_abs_c(cplx{v.re.hi, v.im.hi}));
        st = max(st, __ldcg(P.pst + d.item0 + k));
      }
      acc = warp_sum_ddc(acc);
      aux = cert ? warp_sum_ru(aux) : warp_sum_d(aux);
      if (cert) mag = warp_sum_ru(mag);
#pragma unroll
      for (int m = 16; m > 0; m >>= 1) st = max(st, __shfl_xor_sync(0xffffffffu, st, m));
      if (lane == 0) {
        cplx v = ddc_to_c(acc);
        const int fn = ft_fn(d.ft);
        if (fn == kFnPerm && d.dim > 0) {
          const double sc = ldexp(1.0, -(d.dim - 1));  // 1 / 2^(n-1), exact
          v = cscale(v, sc);
          if (!cert) aux *= sc;
        }
        if (cert) {
          // double-word summation of the partials (relative error < 2^-100 per step,
          // d.nitems + 5 steps) plus the final rounding to binary64
          const double dsum = ru_mul(ru_mul((double)(d.nitems + 6), 7.888609052210118e-31), mag);
          aux = ru_add(aux, dsum);
          if (fn == kFnPerm) aux = ru_mul(aux, ldexp(1.0, -(d.dim - 1)));  // v is already scaled
          aux = ru_add(aux, ru_add(ru_mul(kUc, ru_abs_c(v)), kUfl));
          if (!isfinite(aux)) st = max(st, (int)kStUncertified);
        }
        if (st != kStOk) { v = mkc(NAN, NAN); if (cert) aux = INFINITY; }
        P.out[2 * (size_t)w.inst] = v.re;
        P.out[2 * (size_t)w.inst + 1] = v.im;
        P.aux_out[w.inst] = aux;
        P.st_out[w.inst] = st;
      }
    }
  }
}

// ------------------------------------------------------------------ launch helpers
template <unsigned BR>
inline cudaError_t ensure_smem_br(size_t smem) {
  // the kernel's dynamic shared-memory limit only grows; once it is high enough no
  // attribute call is made, so a launch inside a stream capture issues none
  // (per device: the attribute belongs to the device's context).  The function has
  // external linkage so that every translation unit that launches
  // gbs_items_kernel<BR> (the linker keeps one copy of the kernel's host stub) shares
  // ONE record: a per-unit record let one unit lower the limit below what another
  // unit had set and still believed in force.
  constexpr int kDevs = 64;
  static std::atomic<size_t> smem_set[kDevs];
  static std::mutex mu;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kDevs) dev = 0;
  if (smem <= smem_set[dev].load()) return cudaSuccess;
  std::lock_guard<std::mutex> lk(mu);
  if (smem <= smem_set[dev].load()) return cudaSuccess;
  const cudaError_t e =
      cudaFuncSetAttribute(gbs_items_kernel<BR>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e == cudaSuccess) smem_set[dev].store(smem);
  return e;
}

template <unsigned BR>
static cudaError_t launch_br(const ItemLaunch& P, int grid, int warps, cudaStream_t stream) {
  const size_t smem = (size_t)warps * P.ws_doubles * sizeof(double);
  const cudaError_t e = ensure_smem_br<BR>(smem);
  if (e != cudaSuccess) return e;
  gbs_items_kernel<BR><<<grid, warps * 32, smem, stream>>>(P);
  return cudaGetLastError();
}

template <unsigned BR>
static int occ_br(const ItemLaunch& P, int warps) {
  const size_t smem = (size_t)warps * P.ws_doubles * sizeof(double);
  if (ensure_smem_br<BR>(smem) != cudaSuccess) return 0;
  int nb = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, gbs_items_kernel<BR>, warps * 32, smem) != cudaSuccess)
    return 0;
  return nb;
}

// One translation unit per group of branch sets (parallel builds): each defines
//   bool items_launch_<group>(unsigned br, const ItemLaunch&, int grid, int warps, cudaStream_t, cudaError_t*)
//   int  items_occ_<group>(unsigned br, const ItemLaunch&, int warps)        (-1: not in group)
#define GBSB_DEFINE_GROUP(NAME, LIST)                                                              \
  bool items_launch_##NAME(unsigned br, const ItemLaunch& P, int grid, int warps, cudaStream_t s,    \
                           cudaError_t* err) {                                                       \
    switch (br) { LIST(GBSB_LCASE) default: return false; }                                          \
  }                                                                                                  \
  int items_occ_##NAME(unsigned br, const ItemLaunch& P, int warps) {                                \
    switch (br) { LIST(GBSB_OCASE) default: return -1; }                                             \
  }
#define GBSB_LCASE(B) \
  case (unsigned)(B): *err = launch_br<(B)>(P, grid, warps, s); return true;
#define GBSB_OCASE(B) \
  case (unsigned)(B): return occ_br<(B)>(P, warps);

}  // namespace gbsb
