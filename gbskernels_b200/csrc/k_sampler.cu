// k_sampler.cu -- the resident sampler chain: per mode k the conditional
// submatrices of every draw are gathered on the device from the reduced matrix A_k
// and the draws' photon-count prefixes, their hafnians evaluated by the work-item
// kernel (one work item per conditional, the queue planned on the device), and the
// next photon count drawn by inverse CDF from a counter-based random stream -- no
// host round trip between modes; only the final counts are read back.  Each
// conditional hafnian is split into work items of 2^7 subsets (the planner's split)
// by a one-block scan on the device, which also writes the item count the
// work-item kernel reads: large conditionals spread over many warps.
// Reference counterpart: core/sampler_gather.cu:20-57 (index rule), core/sampler_draw.cu
// :15-47 (clip(Re haf, 0) / j! -> normalise -> inverse CDF), core/sampler_session.cu
// :66-137 (the chain), sampling/sampler.py:214-244 (the host side: A_k and 1/j!).
// The draw uses cuRAND's Philox4_32_10 stream per draw (subsequence = draw index), so
// samples are distributionally, not bit-for-bit, equal to a host sampler's.
#include <cuda_runtime.h>
#include <curand_kernel.h>

#include <algorithm>
#include <cstdint>
#include <mutex>
#include <string>
#include <vector>

#include "gbs_items.cuh"

namespace gbsb {

constexpr int kSamplerMaxN = 32;  // the hafnian path's cap (2 M cutoff <= 32)

// One thread per (draw, candidate j): the index list of the host sampler,
//   [mode i x prefix[i]] + [mode k-1 x j] + [mode i+k x prefix[i]] + [mode 2k-1 x j],
// and the compact n x n submatrix A_k[idx, idx] at the slot of the instance, with the
// instance's descriptor (its work items are assigned by sampler_plan_kernel).
// With `urep` (the prefixes deduplicated, see sampler_key_kernel): instance t is
// candidate j of unique prefix t / (cutoff + 1), read from its representative draw
// urep[u]; instances past *nuniq x (cutoff + 1) are not written.
__global__ void __launch_bounds__(128) sampler_gather_kernel(const double* __restrict__ Ak, int k,
                                                             const int* __restrict__ state, int M, int d0,
                                                             int ndraw, int cutoff, int slot, double* __restrict__ sub,
                                                             InstDesc* __restrict__ insts, int* __restrict__ overflow,
                                                             const int* __restrict__ urep,
                                                             const int* __restrict__ nuniq) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= ndraw * (cutoff + 1)) return;
  const int u = t / (cutoff + 1), j = t % (cutoff + 1);
  if (urep && u >= *nuniq) return;
  const int d = urep ? urep[u] : d0 + u;
  const int* pre = state + (size_t)d * M;
  const int twok = 2 * k;
  int idx[kSamplerMaxN];
  int n = 0;
  bool over = false;
  auto push = [&](int v, int times) {
    for (int r = 0; r < times; ++r) {
      if (n < kSamplerMaxN) idx[n++] = v;
      else over = true;
    }
  };
  for (int i = 0; i < k - 1; ++i) push(i, pre[i]);
  push(k - 1, j);
  for (int i = 0; i < k - 1; ++i) push(i + k, pre[i]);
  push(twok - 1, j);
  if (n > slot) over = true;
  if (over) {
    atomicExch(overflow, 1);
    n = 0;
  }
  double2* out = reinterpret_cast<double2*>(sub + (size_t)t * slot * slot * 2);
  const double2* A = reinterpret_cast<const double2*>(Ak);
  if (n == 0) {
    // haf of the empty matrix is 1: evaluated as haf([[0, 1], [1, 0]]) = 1 (exact)
    out[0] = make_double2(0.0, 0.0);
    out[1] = make_double2(1.0, 0.0);
    out[2] = make_double2(1.0, 0.0);
    out[3] = make_double2(0.0, 0.0);
    n = 2;
  } else {
    for (int r = 0; r < n; ++r)
      for (int c = 0; c < n; ++c) out[r * n + c] = A[(size_t)idx[r] * twok + idx[c]];
  }
  InstDesc D{};
  D.off = (long long)t * slot * slot * 2;
  D.dim = n;
  D.ft = ft_code(kFnHaf, kTierFp64);
  D.item0 = 0;
  D.nitems = 0;
  D.param = 0;
  D.real_in = 0;
  insts[t] = D;
}

// One block: every instance's work items -- 2^min(n/2, 7) subsets each, in subset
// order, as the planner splits a hafnian -- at consecutive indices (exclusive scan
// over the instances in order), and the total item count for the work-item kernel.
constexpr int kSamplerPlanThreads = 1024;
__global__ void __launch_bounds__(kSamplerPlanThreads) sampler_plan_kernel(InstDesc* __restrict__ insts, int ni,
                                                                           WorkItem* __restrict__ items,
                                                                           int* __restrict__ n_items,
                                                                           const int* __restrict__ nuniq, int per_u) {
  __shared__ long long part[kSamplerPlanThreads];
  const int tid = threadIdx.x;
  if (nuniq) ni = min(ni, *nuniq * per_u);  // deduplicated prefixes: the unique instances only
  const int per = (ni + kSamplerPlanThreads - 1) / kSamplerPlanThreads;
  const int t0 = min(ni, tid * per), t1 = min(ni, t0 + per);
  auto splits = [&](int t) -> long long {
    const int h = insts[t].dim / 2;
    return h > kHafItemLog2 ? (1ll << (h - kHafItemLog2)) : 1;
  };
  long long mine = 0;
  for (int t = t0; t < t1; ++t) mine += splits(t);
  part[tid] = mine;
  __syncthreads();
  // inclusive scan of the thread sums (Hillis-Steele in shared memory)
  for (int off = 1; off < kSamplerPlanThreads; off <<= 1) {
    const long long v = tid >= off ? part[tid - off] : 0;
    __syncthreads();
    part[tid] += v;
    __syncthreads();
  }
  long long base = part[tid] - mine;
  for (int t = t0; t < t1; ++t) {
    const int h = insts[t].dim / 2;
    const int lg = h < kHafItemLog2 ? h : kHafItemLog2;
    const long long ns = splits(t);
    insts[t].item0 = (int)base;
    insts[t].nitems = (int)ns;
    for (long long q = 0; q < ns; ++q) {
      WorkItem w{};
      w.inst = t;
      w.lo = (unsigned long long)q << lg;
      w.count = 1ull << lg;
      items[base + q] = w;
    }
    base += ns;
  }
  if (tid == kSamplerPlanThreads - 1) *n_items = (int)part[tid];
}

// One thread per draw: weights clip(Re haf_j, 0) / j!, normalised, inverse CDF with
// one uniform from the draw's stream; the count goes to state[d][k-1].
__global__ void __launch_bounds__(128) sampler_draw_kernel(const double* __restrict__ haf, const double* __restrict__ invfac,
                                                           int cutoff, int d0, int ndraw, unsigned long long seed, int k,
                                                           int* __restrict__ state, int M,
                                                           const int* __restrict__ slot_of,
                                                           const int* __restrict__ sid) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= ndraw) return;
  const int d = d0 + t;
  const int u = slot_of ? sid[slot_of[t]] : t;  // the draw's (unique) prefix
  const double* w = haf + (size_t)u * (cutoff + 1) * 2;  // complex values, real parts used
  double sum = 0.0;
  for (int j = 0; j <= cutoff; ++j) sum += fmax(w[2 * j], 0.0) * invfac[j];
  int photon = 0;
  if (sum > 0.0) {
    // stream of draw d, one uniform per mode: subsequence d, offset k - 1
    curandStatePhilox4_32_10_t st;
    curand_init(seed, (unsigned long long)d, (unsigned long long)(k - 1) * 4ull, &st);
    const double u = curand_uniform_double(&st);
    double c = 0.0;
    for (int j = 0; j <= cutoff; ++j) {
      c += (fmax(w[2 * j], 0.0) * invfac[j]) / sum;
      if (c < u) ++photon;
    }
  }
  state[(size_t)d * M + (k - 1)] = photon;
}

// ---- prefix deduplication.  The conditional hafnians of mode k depend on a draw
// only through its prefix (the counts of modes 1..k-1), and with few photons many
// of the draws share one: at M = 8 and cutoff 2 there are at most 3^7 = 2187
// prefixes at the last mode against 10^5 draws.  Each prefix is a mixed-radix key
// (radix cutoff + 1, used only when (cutoff + 1)^(M - 1) < 2^62), inserted into an
// open-addressing table (linear probing, at least twice as many slots as draws);
// the occupied slots are numbered by one scan, and every unique prefix is gathered
// and evaluated once.  A hafnian does not depend on which instance slot holds it,
// so the draws are bit-identical to evaluating every draw's conditionals.
constexpr unsigned long long kSamplerEmpty = ~0ull;

__device__ __forceinline__ unsigned long long sampler_mix(unsigned long long x) {
  // SplitMix64 finaliser (Steele, Lea, Flood 2014): spreads nearby keys over the table
  x ^= x >> 30;
  x *= 0xbf58476d1ce4e5b9ull;
  x ^= x >> 27;
  x *= 0x94d049bb133111ebull;
  x ^= x >> 31;
  return x;
}

// One thread per draw: insert the prefix key; record the draw's table slot and, for
// the first draw of a key, that draw as the key's representative.  The probe visits
// each slot at most once (the table has more slots than draws, so it always ends).
__global__ void __launch_bounds__(128) sampler_key_kernel(const int* __restrict__ state, int M, int d0, int ndraw,
                                                          int k, int radix, unsigned long long* __restrict__ tkeys,
                                                          int* __restrict__ trep, int tmask,
                                                          int* __restrict__ slot_of) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= ndraw) return;
  const int d = d0 + t;
  const int* pre = state + (size_t)d * M;
  unsigned long long key = 0, mul = 1;
  for (int i = 0; i < k - 1; ++i) {
    key += (unsigned long long)pre[i] * mul;
    mul *= (unsigned long long)radix;
  }
  unsigned int h = (unsigned int)(sampler_mix(key) & (unsigned long long)tmask);
  for (int probe = 0; probe <= tmask; ++probe) {
    const unsigned long long prev = atomicCAS(tkeys + h, kSamplerEmpty, key);
    if (prev == kSamplerEmpty) {
      trep[h] = d;
      break;
    }
    if (prev == key) break;
    h = (h + 1) & (unsigned int)tmask;
  }
  slot_of[t] = (int)h;
}

// One block: number the occupied slots in slot order (sid[slot], -1 when empty), the
// representatives urep[id] and the count *nuniq.
__global__ void __launch_bounds__(kSamplerPlanThreads) sampler_compact_kernel(
    const unsigned long long* __restrict__ tkeys, const int* __restrict__ trep, int tsize, int* __restrict__ sid,
    int* __restrict__ urep, int* __restrict__ nuniq) {
  __shared__ int part[kSamplerPlanThreads];
  const int tid = threadIdx.x;
  const int per = (tsize + kSamplerPlanThreads - 1) / kSamplerPlanThreads;
  const int h0 = min(tsize, tid * per), h1 = min(tsize, h0 + per);
  int mine = 0;
  for (int h = h0; h < h1; ++h) mine += tkeys[h] != kSamplerEmpty;
  part[tid] = mine;
  __syncthreads();
  for (int off = 1; off < kSamplerPlanThreads; off <<= 1) {
    const int v = tid >= off ? part[tid - off] : 0;
    __syncthreads();
    part[tid] += v;
    __syncthreads();
  }
  int id = part[tid] - mine;
  for (int h = h0; h < h1; ++h) {
    if (tkeys[h] != kSamplerEmpty) {
      sid[h] = id;
      urep[id] = trep[h];
      ++id;
    } else {
      sid[h] = -1;
    }
  }
  if (tid == kSamplerPlanThreads - 1) *nuniq = part[tid];
}

bool g_sampler_dedup = true;  // gbs_sampler_set_dedup

namespace {
thread_local std::string t_sampler_err;
int sampler_fail(int code, const std::string& msg) {
  t_sampler_err = msg;
  return code;
}

// Device buffers of the chain, kept per device between calls and grown only when a
// call needs more: allocating and freeing them per call (cudaFree synchronises the
// device) cost more host time than the chain's kernels on 100,000 draws, and made
// the call time vary several-fold from run to run.  Calls hold g_sampler_mu.
template <typename T>
struct DevBuf {
  T* p = nullptr;
  size_t cap = 0;
  cudaError_t need(size_t n) {
    n = std::max<size_t>(n, 1);
    if (n <= cap) return cudaSuccess;
    if (p) cudaFree(p);
    p = nullptr;
    cap = 0;
    const cudaError_t e = cudaMalloc(&p, sizeof(T) * n);
    if (e == cudaSuccess) cap = n;
    return e;
  }
};
struct SamplerBufs {
  DevBuf<double> Ak, invfac, sub, part, paux, out, aux;
  DevBuf<int> state, head, done, pst, st, overflow;
  DevBuf<InstDesc> insts;
  DevBuf<WorkItem> items;
  // prefix deduplication: the table (keys, representative draw, slot number), each
  // draw's slot, the unique prefixes' representatives and their count
  DevBuf<unsigned long long> tkeys;
  DevBuf<int> trep, sid, slot_of, urep, nuniq;
};
constexpr int kSamplerDevs = 64;
SamplerBufs g_sampler[kSamplerDevs];
std::mutex g_sampler_mu;

// The chain over modes 1..M for draws [0, num_draws), in chunks whose conditional
// submatrices fit the slot budget.  weights_out (optional, testing): the Re(haf)
// of every (draw, j) at mode k_weights instead of drawing there.
int sampler_chain(const double* h_Ak, long long ak_total, const int* h_off, int M, int num_draws, int cutoff,
                  const double* h_invfac, unsigned long long seed, int* h_out, int k_stop, const int* h_state_in,
                  double* weights_out) {
  if (M <= 0 || num_draws < 0 || cutoff < 0) return sampler_fail((int)cudaErrorInvalidValue, "sampler: bad sizes");
  if (num_draws == 0) return 0;
  if (!h_Ak || !h_off || (!h_invfac && !weights_out) || (!h_out && !weights_out))
    return sampler_fail((int)cudaErrorInvalidValue, "sampler: null pointer");
  std::vector<double> ones;
  if (!h_invfac) {
    ones.assign((size_t)cutoff + 1, 1.0);
    h_invfac = ones.data();
  }
  if (2 * M * cutoff > kSamplerMaxN)
    return sampler_fail((int)cudaErrorInvalidValue,
                        "sampler: the worst-case conditional submatrix 2 M cutoff exceeds the hafnian cap 32");
  for (int k = 1; k <= M; ++k)
    if (h_off[k - 1] < 0 || (long long)h_off[k - 1] + 4ll * k * k > ak_total)
      return sampler_fail((int)cudaErrorInvalidValue, "sampler: A_k offsets outside the buffer");
  std::lock_guard<std::mutex> lk(g_sampler_mu);
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kSamplerDevs)
    return sampler_fail((int)cudaErrorInvalidDevice, "sampler: no usable device");
  SamplerBufs& B = g_sampler[dev];
  if (B.overflow.p) {
    // a device reset (cudaDeviceReset) since the last call frees every allocation:
    // the cached pointers then no longer name device memory, and are dropped
    cudaPointerAttributes pa{};
    if (cudaPointerGetAttributes(&pa, B.overflow.p) != cudaSuccess || pa.type != cudaMemoryTypeDevice) {
      cudaGetLastError();
      B = SamplerBufs{};
    }
  }
  const int per = cutoff + 1;
  const int slot_max = std::max(2, std::min(kSamplerMaxN, 2 * M * cutoff));
  // work items per instance at most (2^7 subsets each)
  const size_t max_split = (size_t)1 << std::max(0, slot_max / 2 - kHafItemLog2);
  // the slots and item arrays of one step's instances stay within 1 GiB
  const size_t draw_bytes = (size_t)per * ((size_t)slot_max * slot_max * 16 +
                                           max_split * (sizeof(WorkItem) + 4 * sizeof(double) + sizeof(double) + sizeof(int)));
  const size_t fit = std::max<size_t>(1, (size_t)(1ull << 30) / draw_bytes);  // prefixes whose instances fit
  // prefix deduplication when sampling and every prefix key fits: (cutoff + 1)^(M - 1) < 2^62
  bool dedup = g_sampler_dedup && !weights_out;
  long double span = 1.0L;  // distinct prefixes at the last mode at most
  for (int i = 0; i < M - 1 && dedup; ++i) {
    span *= (long double)per;
    if (span >= 4.611686018427387904e18L) dedup = false;
  }
  // draws per chunk and distinct prefixes per step: without deduplication every draw
  // has its own instances; with it the instances follow the distinct prefixes, so
  // when they all fit a chunk can hold up to 2^22 draws (its table and slots alone)
  int chunk, ucap;
  if (dedup && span <= (long double)fit) {
    chunk = (int)std::min<long long>(num_draws, 1ll << 22);
    ucap = (int)std::min<long double>((long double)chunk, span);
  } else {
    chunk = (int)std::min<size_t>(num_draws, fit);
    ucap = chunk;
  }
  const int ninst = ucap * per;
  const size_t nitem_cap = (size_t)ninst * max_split;
  if (nitem_cap > (size_t)INT32_MAX) return sampler_fail((int)cudaErrorInvalidValue, "sampler: too many work items");
  cudaError_t e = B.Ak.need(2 * (size_t)std::max<long long>(ak_total, 1));
  if (e == cudaSuccess) e = B.invfac.need(per);
  if (e == cudaSuccess) e = B.sub.need((size_t)ninst * slot_max * slot_max * 2);
  if (e == cudaSuccess) e = B.part.need(4 * nitem_cap);
  if (e == cudaSuccess) e = B.paux.need(nitem_cap);
  if (e == cudaSuccess) e = B.out.need(2 * (size_t)ninst);
  if (e == cudaSuccess) e = B.aux.need(ninst);
  if (e == cudaSuccess) e = B.state.need((size_t)num_draws * M);
  if (e == cudaSuccess) e = B.head.need(2);  // queue head, item count
  if (e == cudaSuccess) e = B.done.need(ninst);
  if (e == cudaSuccess) e = B.pst.need(nitem_cap);
  if (e == cudaSuccess) e = B.st.need(ninst);
  if (e == cudaSuccess) e = B.overflow.need(1);
  if (e == cudaSuccess) e = B.insts.need(ninst);
  if (e == cudaSuccess) e = B.items.need(nitem_cap);
  int tsize = 1;
  while (tsize < 2 * chunk) tsize <<= 1;
  if (dedup && e == cudaSuccess) e = B.tkeys.need(tsize);
  if (dedup && e == cudaSuccess) e = B.trep.need(tsize);
  if (dedup && e == cudaSuccess) e = B.sid.need(tsize);
  if (dedup && e == cudaSuccess) e = B.slot_of.need(chunk);
  if (dedup && e == cudaSuccess) e = B.urep.need(chunk);
  if (dedup && e == cudaSuccess) e = B.nuniq.need(1);
  if (e != cudaSuccess) return sampler_fail((int)e, "sampler: device allocation failed");
  cudaStream_t s = nullptr;
  e = cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking);
  if (e != cudaSuccess) return sampler_fail((int)e, "sampler: stream");
  e = cudaMemcpyAsync(B.Ak.p, h_Ak, sizeof(double) * 2 * ak_total, cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess) e = cudaMemcpyAsync(B.invfac.p, h_invfac, sizeof(double) * per, cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess) {
    if (h_state_in)
      e = cudaMemcpyAsync(B.state.p, h_state_in, sizeof(int) * (size_t)num_draws * M, cudaMemcpyHostToDevice, s);
    else
      e = cudaMemsetAsync(B.state.p, 0, sizeof(int) * (size_t)num_draws * M, s);
  }
  if (e == cudaSuccess) e = cudaMemsetAsync(B.overflow.p, 0, sizeof(int), s);
  // the hafnian launch: one-warp blocks, the grid from the occupancy of the kernel
  constexpr unsigned BR = br1(kFnHaf, kTierFp64);
  ItemLaunch L{};
  L.mats = B.sub.p;
  L.insts = B.insts.p;
  L.items = B.items.p;
  L.order = nullptr;
  L.head = B.head.p;
  L.done = B.done.p;
  L.part = B.part.p;
  L.paux = B.paux.p;
  L.pst = B.pst.p;
  L.out = B.out.p;
  L.aux_out = B.aux.p;
  L.st_out = B.st.p;
  L.n_items_dev = B.head.p + 1;
  L.haf_smax = slot_max;
  L.ws_doubles = (haf_layout(slot_max).total + 3) & ~3;
  int sms = 0;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const int bps = occ_br<BR>(L, 1);
  if (bps <= 0) {
    cudaStreamDestroy(s);
    return sampler_fail((int)cudaErrorInvalidConfiguration, "sampler: hafnian kernel does not fit");
  }
  // sampling: modes 1..M; weights only: mode k_stop on the given prefixes
  const int kmax = k_stop > 0 ? k_stop : M;
  const int kfirst = weights_out ? kmax : 1;
  for (int d0 = 0; d0 < num_draws && e == cudaSuccess; d0 += chunk) {
    const int nd = std::min(chunk, num_draws - d0);
    const int ni = nd * per;
    for (int k = kfirst; k <= kmax && e == cudaSuccess; ++k) {
      const int slot = std::max(2, std::min(kSamplerMaxN, 2 * k * cutoff));
      if (dedup) {
        e = cudaMemsetAsync(B.tkeys.p, 0xFF, sizeof(unsigned long long) * tsize, s);
        if (e == cudaSuccess) {
          sampler_key_kernel<<<(nd + 127) / 128, 128, 0, s>>>(B.state.p, M, d0, nd, k, per, B.tkeys.p, B.trep.p, tsize - 1,
                                                              B.slot_of.p);
          e = cudaGetLastError();
        }
        if (e == cudaSuccess) {
          sampler_compact_kernel<<<1, kSamplerPlanThreads, 0, s>>>(B.tkeys.p, B.trep.p, tsize, B.sid.p, B.urep.p, B.nuniq.p);
          e = cudaGetLastError();
        }
        if (e != cudaSuccess) break;
      }
      sampler_gather_kernel<<<(ni + 127) / 128, 128, 0, s>>>(B.Ak.p + 2 * (size_t)h_off[k - 1], k, B.state.p, M, d0, nd,
                                                            cutoff, slot, B.sub.p, B.insts.p, B.overflow.p,
                                                            dedup ? B.urep.p : nullptr, dedup ? B.nuniq.p : nullptr);
      e = cudaGetLastError();
      if (e == cudaSuccess) {
        sampler_plan_kernel<<<1, kSamplerPlanThreads, 0, s>>>(B.insts.p, ni, B.items.p, B.head.p + 1,
                                                             dedup ? B.nuniq.p : nullptr, per);
        e = cudaGetLastError();
      }
      if (e == cudaSuccess) e = cudaMemsetAsync(B.head.p, 0, sizeof(int), s);
      if (e == cudaSuccess) e = cudaMemsetAsync(B.done.p, 0, sizeof(int) * std::min(ni, ninst), s);
      if (e == cudaSuccess) {
        L.n_items = (int)nitem_cap;  // upper bound; the kernel reads the planned count
        e = launch_br<BR>(L, sms * bps, 1, s);
      }
      if (e != cudaSuccess) break;
      if (weights_out && k == kmax) {
        std::vector<double> o(2 * (size_t)ni);
        e = cudaMemcpyAsync(o.data(), B.out.p, sizeof(double) * 2 * ni, cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
        for (int t = 0; t < ni && e == cudaSuccess; ++t) weights_out[(size_t)d0 * per + t] = o[2 * (size_t)t];
        break;
      }
      sampler_draw_kernel<<<(nd + 127) / 128, 128, 0, s>>>(B.out.p, B.invfac.p, cutoff, d0, nd, seed, k, B.state.p, M,
                                                           dedup ? B.slot_of.p : nullptr, dedup ? B.sid.p : nullptr);
      e = cudaGetLastError();
    }
  }
  int over = 0;
  if (e == cudaSuccess) e = cudaMemcpyAsync(&over, B.overflow.p, sizeof(int), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess && h_out)
    e = cudaMemcpyAsync(h_out, B.state.p, sizeof(int) * (size_t)num_draws * M, cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  cudaStreamDestroy(s);
  if (e != cudaSuccess) return sampler_fail((int)e, std::string("sampler: ") + cudaGetErrorString(e));
  if (over) return sampler_fail((int)cudaErrorInvalidValue, "sampler: a conditional submatrix exceeded its slot");
  return 0;
}
}  // namespace

}  // namespace gbsb

using namespace gbsb;

extern "C" {

// h_Ak: the M reduced A-matrices concatenated (A_k is 2k x 2k complex row-major,
// starting at complex element h_off[k-1]); ak_total complex elements.  h_out:
// num_draws x M photon counts (row-major).  maxn is accepted for the reference's
// signature; the slot of mode k is 2 k cutoff (<= 32, checked).
int gbs_sampler_sample(const double* h_Ak, int ak_total, const int* h_off, int M, int num_draws, int cutoff,
                       int maxn, const double* h_invfac, unsigned long long seed, int* h_out) {
  (void)maxn;
  return sampler_chain(h_Ak, ak_total, h_off, M, num_draws, cutoff, h_invfac, seed, h_out, 0, nullptr, nullptr);
}

// Prefix deduplication of the sampler chain on (1, default) or off (0): every draw's
// conditional hafnians evaluated separately.  The samples are the same either way;
// the switch exists to check that.  Process-wide.
int gbs_sampler_set_dedup(int on) {
  g_sampler_dedup = on != 0;
  return 0;
}

// The conditional weights Re haf(A_k[idx, idx]) of mode k for given prefixes
// (h_state: num_draws x M counts, columns < k - 1 used): num_draws x (cutoff + 1).
int gbs_sampler_conditional_weights(const double* h_Ak, int ak_total, const int* h_off, int M, int k,
                                    const int* h_state, int num_draws, int cutoff, double* h_w) {
  if (k < 1 || k > M) return sampler_fail((int)cudaErrorInvalidValue, "sampler: mode index out of range");
  if (!h_state || !h_w) return sampler_fail((int)cudaErrorInvalidValue, "sampler: null pointer");
  return sampler_chain(h_Ak, ak_total, h_off, M, num_draws, cutoff, nullptr, 0, nullptr, k, h_state, h_w);
}

const char* gbs_sampler_last_error(void) { return t_sampler_err.c_str(); }

}  // extern "C"
