// host_api.cu -- the C++ host runtime and the C ABI of libgbs_b200.so.
//
// Layers (each replaces a reference component; citations are to the reference):
//   * planner: cuts every instance into work items (function of (func, tier, size)
//     only, so values are independent of batch composition);
//   * session: stream + monotonically growing device buffers + pinned staging
//     (core/host_api.cu:474-648, gbs_session_*), one H2D of the packed batch, one
//     launch, one D2H;
//   * bucketing: the ragged "plain per-size launch" path, one launch per
//     (func, tier, size) bucket (gbskernels/__init__.py:813-852 Workspace._ragged);
//   * persistent mixed queue: ONE launch over all instances of a ragged, mixed
//     function / tier batch, work items ordered heaviest first (new);
//   * tier logic: auto = fp64 + sum|term| indicator, device double-double rerun of
//     the elements with kappa >= 1e8 (gbskernels/__init__.py:240-297, without the
//     reference's CPU mpmath fallback);
//   * C ABI: gbs_*_host, gbs_session_*, gbs_queue_* (include/gbs_b200.h).
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "gbs_kernels.cuh"
#include "haf_dd.cuh"
#include "haf_pt.cuh"
#include "tor_lu.cuh"
#include "tor_warp.cuh"
#include "tor_warp_dd.cuh"

namespace gbsb {

// kernel groups (k_*.cu)
#define GBSB_DECL_GROUP(NAME)                                                                       \
  bool items_launch_##NAME(unsigned br, const ItemLaunch& P, int grid, int warps, cudaStream_t s,   \
                           cudaError_t* err);                                                       \
  int items_occ_##NAME(unsigned br, const ItemLaunch& P, int warps);
GBSB_DECL_GROUP(perm_fp64)
GBSB_DECL_GROUP(perm_kappa)
GBSB_DECL_GROUP(perm_dd)
GBSB_DECL_GROUP(haf)
GBSB_DECL_GROUP(haf_dd)
GBSB_DECL_GROUP(tor)
GBSB_DECL_GROUP(mixed)
GBSB_DECL_GROUP(perm_cert)
GBSB_DECL_GROUP(cert)
#undef GBSB_DECL_GROUP

static cudaError_t launch_any(unsigned br, const ItemLaunch& P, int grid, int warps, cudaStream_t s) {
  cudaError_t e = cudaErrorInvalidValue;
  if (items_launch_perm_fp64(br, P, grid, warps, s, &e)) return e;
  if (items_launch_perm_kappa(br, P, grid, warps, s, &e)) return e;
  if (items_launch_perm_dd(br, P, grid, warps, s, &e)) return e;
  if (items_launch_haf(br, P, grid, warps, s, &e)) return e;
  if (items_launch_haf_dd(br, P, grid, warps, s, &e)) return e;
  if (items_launch_tor(br, P, grid, warps, s, &e)) return e;
  if (items_launch_mixed(br, P, grid, warps, s, &e)) return e;
  if (items_launch_perm_cert(br, P, grid, warps, s, &e)) return e;
  if (items_launch_cert(br, P, grid, warps, s, &e)) return e;
  return cudaErrorInvalidValue;
}
static int occ_any(unsigned br, const ItemLaunch& P, int warps) {
  int r;
  if ((r = items_occ_perm_fp64(br, P, warps)) >= 0) return r;
  if ((r = items_occ_perm_kappa(br, P, warps)) >= 0) return r;
  if ((r = items_occ_perm_dd(br, P, warps)) >= 0) return r;
  if ((r = items_occ_haf(br, P, warps)) >= 0) return r;
  if ((r = items_occ_haf_dd(br, P, warps)) >= 0) return r;
  if ((r = items_occ_tor(br, P, warps)) >= 0) return r;
  if ((r = items_occ_mixed(br, P, warps)) >= 0) return r;
  if ((r = items_occ_perm_cert(br, P, warps)) >= 0) return r;
  if ((r = items_occ_cert(br, P, warps)) >= 0) return r;
  return 0;
}
// Smallest compiled branch set covering `need`.
static unsigned cover(unsigned need) {
  if (__builtin_popcount(need) == 1) return need;
  const unsigned sets[] = {kBrHafLhafFp64, kBrServe, kBrMixed};
  for (unsigned s : sets)
    if ((s & need) == need) return s;
  return 0;  // not coverable by one launch (the caller splits)
}

// ------------------------------------------------------------------ caps
constexpr int kPermCap = 28;
constexpr int kHafCap = kHafMaxN;   // 32 (after odd-N loop augmentation)
constexpr int kTorCapModes = 24;        // batched torontonian
constexpr int kTorSingleCapModes = 32;  // single-large torontonian (binary64 tiers)

// ------------------------------------------------------------------ requests and plans
struct Req {
  int fn, tier;
  int dim;              // matrix side as given by the caller (tor: 2n)
  const double* mat;    // complex interleaved, row-major (host); null for a state request
  // resident-state request: the matrix is gathered on the device as
  // state[idx[r]][idx[c]] (loop weights gamma[idx[r]] on the diagonal when gamma)
  const double* state = nullptr;  // device, M x M complex
  const double* gamma = nullptr;  // device, M complex (or null)
  const int* idx = nullptr;       // host, dim indices
  int M = 0;
  int state_real = 0;
  // single-large torontonian: the 32-mode cap applies, and the prefix split is at
  // least 2^split work items (the reference's `groups`)
  int single = 0;
  int split = -1;
};

// Device gather of resident-state submatrices (k_gather.cu).
struct GatherDesc {
  long long out_off;   // doubles into the packed matrix buffer
  long long idx_off;   // ints into the index array
  const double* state;
  const double* gamma;
  int d, de, M, use_gamma;
};
cudaError_t launch_gather(const GatherDesc* descs, int n, const int* idx, double* mats, cudaStream_t st);
// Scatter of a plan's results to request order on the device (k_gather.cu).
struct ScatterArgs {
  const double* out;
  const double* aux;
  const int* st;
  const int* map;
  int ni;
  const int* tidx;
  const double* tval;
  int ntriv;
  double* dval;
  double* daux;
  int* dst;
  int write_aux;
};
cudaError_t launch_scatter(const ScatterArgs& a, cudaStream_t st);

struct Plan {
  std::vector<InstDesc> insts;
  std::vector<WorkItem> items;
  std::vector<int> order;
  std::vector<int> trivial;      // instances answered on the host (size-0 / odd haf)
  std::vector<cplx> trivial_val;
  unsigned need = 0;
  int haf_smax = 2;
  int ws_doubles = 0;
  long long mat_doubles = 0;
  double cost = 0.0;
};


// ------------------------------------------------------------------ tuned splits
// Work-item split and block size per (function, binary64 or double-double tiers,
// evaluated side), written by the autotuner through gbs_set_split; 0 = unset (the
// planner's default).  Stored as value + 1.  The binary64 tiers (fp64, indicator,
// certified) share one entry so their values stay bit-identical.
constexpr int kTuneDims = 65;
static std::atomic<int> g_tune_split[4][2][kTuneDims];
static std::atomic<int> g_tune_warps[4][2][kTuneDims];
int tuned_split(int fn, int tier, int dim) {  // also read by the allocation-free entry point
  if (fn < 0 || fn > 3 || dim < 0 || dim >= kTuneDims) return -1;
  return g_tune_split[fn][(tier == kTierDD || tier == kTierCertDD) ? 1 : 0][dim].load() - 1;
}
static int tuned_warps(int fn, int tier, int dim) {
  if (fn < 0 || fn > 3 || dim < 0 || dim >= kTuneDims) return 0;
  return g_tune_warps[fn][(tier == kTierDD || tier == kTierCertDD) ? 1 : 0][dim].load();
}

// Cost model (relative units) used only to order the queue heaviest-first.
static double item_cost(int fn, int dim, unsigned long long count, int tier, int param) {
  double c;
  switch (fn) {
    case kFnPerm: c = (double)count * dim; break;
    case kFnTor: {
      // binary64 tiers: count prefix patterns, 2^(q - g) leaves of 32 subsets each
      // (g = param); double-double: count lanes of 2^(n - g) subsets each
      const int n = dim / 2, q = n - std::min(n, 5);
      if (param < 0) {  // complex O: count subset LU factorisations
        c = (double)count * dim * dim * dim;
        break;
      }
      const int qd = n - std::min(n, 4);
      c = (tier == kTierDD || tier == kTierCertDD) ? 20.0 * (double)count * std::ldexp(1.0, qd - param) * 16.0 * (36.0 * qd + 900.0)
                          : (double)count * std::ldexp(1.0, q - param) * 32.0 * (36.0 * q + 1400.0);
      break;
    }
    default: { double n = dim / 2.0; c = (double)count * (n + 1) * n * n * n; break; }
  }
  return (tier == kTierDD || tier == kTierCertDD) ? 20.0 * c : c;
}

// Append one instance (already validated) to the plan.  Returns the instance index.
static int plan_instance(Plan& P, int fn, int tier, int dim_eval, bool real_in, long long off, int split = -1) {
  InstDesc d{};
  d.off = off;
  d.dim = dim_eval;
  d.ft = ft_code(fn, tier);
  d.item0 = (int)P.items.size();
  d.param = 0;
  d.real_in = real_in ? 1 : 0;
  const int idx = (int)P.insts.size();
  auto add = [&](unsigned long long lo, unsigned long long count) {
    WorkItem w{};
    w.inst = idx;
    w.lo = lo;
    w.count = count;
    P.items.push_back(w);
  };
  if (fn == kFnPerm) {
    const int n = dim_eval;
    const unsigned long long terms = 1ull << (n - 1);
    if (terms <= 32) {
      add(0, terms);
    } else {
      const int rcap = (tier == kTierDD || tier == kTierCertDD) ? 6 : 10;  // the dd tiers share one split
      int rlog = std::min(n - 1 - 5, rcap);
      const int tl = tuned_split(fn, tier, dim_eval);
      if (tl >= 0) rlog = std::min(n - 1 - 5, tl);
      const unsigned long long cnt = 32ull << rlog;
      for (unsigned long long lo = 0; lo < terms; lo += cnt) add(lo, cnt);
      d.param = rlog;
    }
  } else if (fn == kFnHaf || fn == kFnLhaf) {
    const int n = dim_eval / 2;
    const unsigned long long masks = 1ull << n;
    // masks per item: 2^kHafItemLog2 (binary64 tiers) / 2^6 (double-double); smaller instances are one item
    int per = (tier == kTierDD || tier == kTierCertDD) ? std::min(n, 6) : std::min(n, kHafItemLog2);  // dd tiers: one split
    const int tl = tuned_split(fn, tier, dim_eval);
    if (tl >= 0) per = std::min(n, tl);
    const unsigned long long cnt = 1ull << per;
    for (unsigned long long lo = 0; lo < masks; lo += cnt) add(lo, std::min(cnt, masks - lo));
    P.haf_smax = std::max(P.haf_smax, dim_eval);
  } else if (!real_in) {  // tor, complex O: ranges of subset masks, one LU per subset
    const int n = dim_eval / 2;
    const int per = std::min(n, 6);
    for (unsigned long long lo = 0; lo < (1ull << n); lo += (1ull << per)) add(lo, 1ull << per);
    d.param = -1;
  } else if (tier == kTierDD || tier == kTierCertDD) {  // tor, double-double: the warp walk, 16-subset tail
    const int n = dim_eval / 2;
    const int q = n - std::min(n, kTorTailDD);
    int g = std::max(0, q - 6);  // 2^6 prefix leaves per item
    const int tl = tuned_split(fn, tier, dim_eval);
    if (tl >= 0) g = std::max(0, q - tl);
    for (unsigned long long p = 0; p < (1ull << g); ++p) add(p, 1);
    d.param = g;
  } else {  // tor, binary64 tiers: one warp per prefix pattern over the first g prefix modes
    const int n = dim_eval / 2;
    const int q = n - std::min(n, 5);
    // 2^9 leaves (x 32 tail subsets) per item, the same split for every binary64
    // tier so that the certified and indicator values are the fp64 value bit for bit
    int g = std::max(0, q - 9);
    const int tl = tuned_split(fn, tier, dim_eval);  // log2 prefix leaves per item
    if (tl >= 0) g = std::max(0, q - tl);
    if (split >= 0) g = std::min(q, std::max(g, split));
    for (unsigned long long p = 0; p < (1ull << g); ++p) add(p, 1);
    d.param = g;
  }
  d.nitems = (int)P.items.size() - d.item0;
  P.insts.push_back(d);
  P.need |= 1u << d.ft;
  return idx;
}

static int ws_for_plan(const Plan& P) {
  int ws = 2;
  for (const InstDesc& d : P.insts) {
    const int fn = ft_fn(d.ft), tier = ft_tier(d.ft);
    int w = 0;
    if (fn == kFnPerm) w = 2 * d.dim * d.dim;
    else if (fn == kFnTor && !d.real_in) w = tor_lu_ws_doubles(tier == kTierCert);
    else if (fn == kFnTor && (tier == kTierDD || tier == kTierCertDD)) w = tor_d_layout(d.dim / 2, tier == kTierCertDD).total;
    else if (fn == kFnTor) w = tor_w_layout(d.dim / 2, tier == kTierCert).total;
    else if (tier == kTierDD || tier == kTierCertDD) w = haf_dd_layout(P.haf_smax, tier == kTierCertDD).total;
    else if (d.real_in) w = haf_layout(P.haf_smax, tier == kTierCert).total + haf_real_layout(P.haf_smax).total;
    else w = haf_layout(P.haf_smax, tier == kTierCert).total;
    ws = std::max(ws, w);
  }
  return (ws + 3) & ~3;  // 32-byte multiple per warp
}

// ------------------------------------------------------------------ session
struct DevBuf {
  void* p = nullptr;
  size_t cap = 0;
};
struct PinBuf {
  void* p = nullptr;
  size_t cap = 0;
};

}  // namespace gbsb

struct gbs_session {
  cudaStream_t stream = nullptr;
  int device = 0;
  int sms = 148;
  gbsb::DevBuf mats, meta, part, paux, pst, done, head, out, aux, st;
  gbsb::PinBuf pin_in, pin_meta, pin_out;
  gbsb::DevBuf gather;
  gbsb::PinBuf pin_gather;
  gbsb::DevBuf rmap;       // instance -> request map and trivial values of a resident read
  gbsb::PinBuf pin_rmap;
  std::vector<gbsb::GatherDesc> gdesc;
  std::vector<int> gidx;
  size_t reallocs = 0;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  float last_kernel_ms = 0.f;
  int last_launches = 0;
  long long last_items = 0;
  // the current plan (device-resident work queue of the last prepared batch)
  struct Group {
    gbsb::ItemLaunch L;
    unsigned br = 0;
    int grid = 0, warps = 0;
    int ni = 0, nit = 0;
    size_t out_off = 0;     // instance offset into the session's result arrays
    std::vector<int> req;   // request index of each instance
  };
  std::vector<Group> groups;
  int plan_B = 0;
  std::vector<char> plan_trivial;
  std::vector<gbsb::cplx> plan_tval;
  std::vector<int> plan_tier;  // tier of each request
  size_t plan_ninst = 0;
  bool plan_ready = false;
  // CUDA graph of the prepared plan's launch sequence (queue resets + one launch per
  // group), captured on its second run and replayed afterwards; dropped with the plan
  bool use_graphs = true;
  int plan_runs = 0;
  cudaGraphExec_t graph = nullptr;
  std::mutex mu;
};

namespace gbsb {

static thread_local std::string g_last_error;

static int fail(int code, const std::string& msg) {
  g_last_error = msg;
  return code;
}

static cudaError_t grow_dev(DevBuf& b, size_t bytes, size_t* reallocs) {
  if (bytes <= b.cap) return cudaSuccess;
  if (b.p) cudaFree(b.p);
  b.p = nullptr;
  b.cap = 0;
  size_t want = std::max(bytes, (size_t)256);
  cudaError_t e = cudaMalloc(&b.p, want);
  if (e == cudaSuccess) {
    b.cap = want;
    if (reallocs) ++*reallocs;
  }
  return e;
}
static cudaError_t grow_pin(PinBuf& b, size_t bytes) {
  if (bytes <= b.cap) return cudaSuccess;
  if (b.p) cudaFreeHost(b.p);
  b.p = nullptr;
  b.cap = 0;
  size_t want = std::max(bytes, (size_t)256);
  cudaError_t e = cudaMallocHost(&b.p, want);
  if (e == cudaSuccess) b.cap = want;
  return e;
}

// Validate + normalise one request.  Returns 0 or an error code; on success fills
// the evaluated side length (odd loop hafnian augmented) and the real-input flag.
// A hafnian or loop hafnian given as host data with every imaginary part zero runs
// the real power loop in the binary64 tiers (fp64, indicator, certified; the
// double-double walks are complex only).  Resident-state requests stay complex.
static bool haf_real_path(const Req& r) {
  if (r.state || !r.mat) return false;
  if (r.tier != kTierFp64 && r.tier != kTierKappa && r.tier != kTierCert) return false;
  const size_t nn = (size_t)r.dim * r.dim;
  for (size_t i = 0; i < nn; ++i)
    if (r.mat[2 * i + 1] != 0.0) return false;
  return true;
}

static int check_req(const Req& r, int* dim_eval, bool* real_in, bool* trivial, cplx* tval) {
  *trivial = false;
  *real_in = false;
  if (r.dim < 0) return fail(cudaErrorInvalidValue, "negative matrix dimension");
  if (r.tier < 0 || r.tier > 4) return fail(cudaErrorInvalidValue, "unsupported precision tier");

  switch (r.fn) {
    case kFnPerm:
      if (r.dim == 0) { *trivial = true; *tval = mkc(1, 0); return 0; }
      if (r.dim > kPermCap) return fail(cudaErrorInvalidValue, "permanent: n above the cap 28");
      *dim_eval = r.dim;
      return 0;
    case kFnHaf:
      if (r.dim == 0) { *trivial = true; *tval = mkc(1, 0); return 0; }
      if (r.dim & 1) { *trivial = true; *tval = mkc(0, 0); return 0; }
      if (r.dim > kHafCap) return fail(cudaErrorInvalidValue, "hafnian: N above the cap 32");
      *dim_eval = r.dim;
      *real_in = haf_real_path(r);
      return 0;
    case kFnLhaf: {
      if (r.dim == 0) { *trivial = true; *tval = mkc(1, 0); return 0; }
      int d = r.dim + (r.dim & 1);  // lhaf(A) = lhaf(A (+) [1]) for odd N
      if (d > kHafCap) return fail(cudaErrorInvalidValue, "loop hafnian: N above the cap 32");
      *dim_eval = d;
      *real_in = haf_real_path(r);
      return 0;
    }
    case kFnTor: {
      if (r.dim & 1) return fail(cudaErrorInvalidValue, "torontonian: matrix side must be even");
      if (r.dim == 0) { *trivial = true; *tval = mkc(1, 0); return 0; }
      if (r.single) {
        if (r.tier == kTierDD) return fail(cudaErrorNotSupported, "single-large torontonian: no double-double tier");
        if (r.dim / 2 > kTorSingleCapModes)
          return fail(cudaErrorInvalidValue, "single-large torontonian: modes above the cap 32");
      } else if (r.dim / 2 > kTorCapModes) {
        return fail(cudaErrorInvalidValue, "torontonian: modes above the cap 24");
      }
      bool re = true;
      if (r.state) {
        re = r.state_real != 0;
      } else {
        const size_t nn = (size_t)r.dim * r.dim;
        for (size_t i = 0; i < nn; ++i)
          if (r.mat[2 * i + 1] != 0.0) { re = false; break; }
      }
      if (!re) {
        // complex O: subset LU determinants, binary64 tiers, the reference's GPU cap
        if (r.tier == kTierDD || r.tier == kTierCertDD || r.single)
          return fail(cudaErrorNotSupported,
                      "torontonian: complex O is supported in the binary64 tiers only (the double-double "
                      "and single-large paths are real-domain)");
        if (r.dim / 2 > kTorLuMaxModes)
          return fail(cudaErrorInvalidValue, "torontonian: complex O above the cap of 12 modes");
        *real_in = false;
        *dim_eval = r.dim;
        return 0;
      }
      *real_in = true;
      *dim_eval = r.dim;
      return 0;
    }
    default:
      return fail(cudaErrorInvalidValue, "unknown function code");
  }
}

struct RunOpts {
  bool per_size = false;   // one launch per (func, tier, size) bucket
  bool sort_heavy = true;  // heaviest instances first in the queue
  int warps = 4;           // warps per block
};

// Build the device-resident plan of `reqs`: validate, pack and upload every matrix
// once, cut the work items, upload the queue(s).  One group = one launch: a single
// group holds every haf / lhaf / tor request (persistent mixed queue); the
// permanent gets one group per tier; per-size mode gives one group per
// (func, tier, size) bucket.
static void drop_graph(gbs_session* s) {
  if (s->graph) cudaGraphExecDestroy(s->graph);
  s->graph = nullptr;
  s->plan_runs = 0;
}

static int plan_build(gbs_session* s, const std::vector<Req>& reqs, const RunOpts& opt) {
  s->plan_ready = false;
  drop_graph(s);
  s->groups.clear();
  const int B = (int)reqs.size();
  s->plan_B = B;
  s->plan_trivial.assign(B, 0);
  s->plan_tval.assign(B, mkc(0, 0));
  s->plan_tier.assign(B, 0);
  for (int i = 0; i < B; ++i) s->plan_tier[i] = reqs[i].tier;
  s->plan_ninst = 0;
  if (B == 0) { s->plan_ready = true; return 0; }
  std::vector<int> dim_eval(B, 0);
  std::vector<char> real_in(B, 0);
  long long mat_doubles = 0;
  for (int i = 0; i < B; ++i) {
    bool re = false, tr = false;
    int rc = check_req(reqs[i], &dim_eval[i], &re, &tr, &s->plan_tval[i]);
    if (rc) {
      g_last_error = "request #" + std::to_string(i) + ": " + g_last_error;
      return rc;
    }
    real_in[i] = re;
    s->plan_trivial[i] = tr;
    if (!tr) mat_doubles += 2ll * dim_eval[i] * dim_eval[i];
  }
  std::vector<std::vector<int>> groups;
  if (opt.per_size) {
    std::vector<long long> keys;
    for (int i = 0; i < B; ++i) {
      if (s->plan_trivial[i]) continue;
      long long key = ((long long)reqs[i].fn * 8 + reqs[i].tier) * 4096 + dim_eval[i];
      size_t g = std::find(keys.begin(), keys.end(), key) - keys.begin();
      if (g == keys.size()) { keys.push_back(key); groups.emplace_back(); }
      groups[g].push_back(i);
    }
  } else {
    groups.resize(6);  // everything but the permanent, then the permanent per tier (0..4)
    for (int i = 0; i < B; ++i) {
      if (s->plan_trivial[i]) continue;
      groups[reqs[i].fn == kFnPerm ? 1 + reqs[i].tier : 0].push_back(i);
    }
  }
  // ---- plans of every group (host) and the sizes of the concatenated device arrays
  std::vector<Plan> plans;
  std::vector<std::vector<int>> greq;
  for (auto& grp : groups) {
    if (grp.empty()) continue;
    plans.emplace_back();
    greq.push_back(grp);
  }
  std::vector<long long> off(B, 0);
  {
    long long o = 0;
    for (int i = 0; i < B; ++i) {
      if (s->plan_trivial[i]) continue;
      off[i] = o;
      o += 2ll * dim_eval[i] * dim_eval[i];
    }
  }
  size_t meta_bytes = 0, tot_items = 0, tot_inst = 0;
  for (size_t g = 0; g < plans.size(); ++g) {
    Plan& P = plans[g];
    for (int i : greq[g]) plan_instance(P, reqs[i].fn, reqs[i].tier, dim_eval[i], real_in[i], off[i], reqs[i].split);
    P.ws_doubles = ws_for_plan(P);
    const int ni = (int)P.insts.size(), nit = (int)P.items.size();
    std::vector<int> inst_order(ni);
    for (int k = 0; k < ni; ++k) inst_order[k] = k;
    if (opt.sort_heavy && !opt.per_size) {
      std::vector<double> c(ni);
      for (int k = 0; k < ni; ++k) {
        const InstDesc& d = P.insts[k];
        c[k] = item_cost(ft_fn(d.ft), d.dim, P.items[d.item0].count, ft_tier(d.ft), d.param);
      }
      std::stable_sort(inst_order.begin(), inst_order.end(), [&](int a, int b) { return c[a] > c[b]; });
    }
    P.order.reserve(nit);
    for (int k : inst_order)
      for (int j = 0; j < P.insts[k].nitems; ++j) P.order.push_back(P.insts[k].item0 + j);
    if (cover(P.need) == 0) return fail(cudaErrorNotSupported, "no compiled kernel covers this mix");
    meta_bytes += ((ni * sizeof(InstDesc) + nit * sizeof(WorkItem) + nit * sizeof(int)) + 255) & ~(size_t)255;
    tot_items += nit;
    tot_inst += ni;
  }
  // ---- buffers (monotone growth)
  cudaError_t e = grow_pin(s->pin_in, std::max<long long>(mat_doubles, 2) * sizeof(double));
  if (e == cudaSuccess) e = grow_dev(s->mats, std::max<long long>(mat_doubles, 2) * sizeof(double), &s->reallocs);
  if (e == cudaSuccess) e = grow_pin(s->pin_meta, std::max<size_t>(meta_bytes, 256));
  if (e == cudaSuccess) e = grow_dev(s->meta, std::max<size_t>(meta_bytes, 256), &s->reallocs);
  if (e == cudaSuccess) e = grow_dev(s->part, std::max<size_t>(tot_items, 1) * 4 * sizeof(double), &s->reallocs);
  if (e == cudaSuccess) e = grow_dev(s->paux, std::max<size_t>(tot_items, 1) * sizeof(double), &s->reallocs);
  if (e == cudaSuccess) e = grow_dev(s->pst, std::max<size_t>(tot_items, 1) * sizeof(int), &s->reallocs);
  if (e == cudaSuccess) e = grow_dev(s->done, std::max<size_t>(tot_inst, 1) * sizeof(int), &s->reallocs);
  if (e == cudaSuccess) e = grow_dev(s->head, 64 * std::max<size_t>(plans.size(), 1), &s->reallocs);
  if (e == cudaSuccess) e = grow_dev(s->out, std::max<size_t>(tot_inst, 1) * 2 * sizeof(double), &s->reallocs);
  if (e == cudaSuccess) e = grow_dev(s->aux, std::max<size_t>(tot_inst, 1) * sizeof(double), &s->reallocs);
  if (e == cudaSuccess) e = grow_dev(s->st, std::max<size_t>(tot_inst, 1) * sizeof(int), &s->reallocs);
  if (e == cudaSuccess) e = grow_pin(s->pin_out, std::max<size_t>(tot_inst, 1) * (3 * sizeof(double) + sizeof(int)));
  if (e != cudaSuccess) return fail(e, "allocating session buffers");
  // staging buffers may still be read by copies of a previous call
  e = cudaStreamSynchronize(s->stream);
  if (e != cudaSuccess) return fail(e, "synchronising the session stream");
  // ---- pack matrices (odd loop hafnians augmented by A (+) [1]) and upload once
  {
    double* dst = (double*)s->pin_in.p;
    s->gdesc.clear();
    s->gidx.clear();
    std::vector<int> host_rows;  // requests copied from host memory
    host_rows.reserve(B);
    for (int i = 0; i < B; ++i) {
      if (s->plan_trivial[i]) continue;
      const int d = reqs[i].dim, de = dim_eval[i];
      if (reqs[i].state) {  // filled on the device by the gather kernel
        GatherDesc gd{off[i], (long long)s->gidx.size(), reqs[i].state, reqs[i].gamma, d, de, reqs[i].M,
                      reqs[i].gamma != nullptr};
        s->gdesc.push_back(gd);
        s->gidx.insert(s->gidx.end(), reqs[i].idx, reqs[i].idx + d);
        continue;
      }
      host_rows.push_back(i);
    }
    auto pack = [&](size_t lo, size_t hi) {
      for (size_t k = lo; k < hi; ++k) {
        const int i = host_rows[k];
        const long long o = off[i];
        const int d = reqs[i].dim, de = dim_eval[i];
        if (de == d) {
          std::memcpy(dst + o, reqs[i].mat, sizeof(double) * 2 * (size_t)d * d);
        } else {
          std::memset(dst + o, 0, sizeof(double) * 2 * (size_t)de * de);
          for (int r = 0; r < d; ++r)
            std::memcpy(dst + o + 2ll * r * de, reqs[i].mat + 2ll * r * d, sizeof(double) * 2 * d);
          dst[o + 2ll * ((long long)d * de + d)] = 1.0;
        }
      }
    };
    // a large batch is packed by several host threads (disjoint ranges of requests,
    // disjoint destination ranges): one thread copies a few GB/s, short of what the
    // upload that follows moves
    const size_t bytes = (size_t)std::max<long long>(mat_doubles, 0) * sizeof(double);
    const int nth = (int)std::min<size_t>({(size_t)std::max(1u, std::thread::hardware_concurrency()), (size_t)8,
                                            bytes / (8u << 20) + 1, host_rows.size() + 1});
    if (nth <= 1) {
      pack(0, host_rows.size());
    } else {
      std::vector<std::thread> th;
      const size_t per = (host_rows.size() + nth - 1) / nth;
      for (int t = 0; t < nth; ++t) {
        const size_t lo = std::min(host_rows.size(), t * per), hi = std::min(host_rows.size(), lo + per);
        if (lo >= hi) continue;
        try {
          th.emplace_back(pack, lo, hi);
        } catch (...) {  // no thread to be had: this range in the calling thread
          pack(lo, hi);
        }
      }
      for (auto& t : th) t.join();
    }
    if (mat_doubles > 0) {
      e = cudaMemcpyAsync(s->mats.p, s->pin_in.p, mat_doubles * sizeof(double), cudaMemcpyHostToDevice, s->stream);
      if (e != cudaSuccess) return fail(e, "uploading matrices");
    }
    if (!s->gdesc.empty()) {
      const size_t gb = s->gdesc.size() * sizeof(GatherDesc), ib = s->gidx.size() * sizeof(int);
      e = grow_pin(s->pin_gather, gb + ib + 64);
      if (e == cudaSuccess) e = grow_dev(s->gather, gb + ib + 64, &s->reallocs);
      if (e != cudaSuccess) return fail(e, "allocating gather descriptors");
      std::memcpy(s->pin_gather.p, s->gdesc.data(), gb);
      std::memcpy((char*)s->pin_gather.p + gb, s->gidx.data(), ib);
      e = cudaMemcpyAsync(s->gather.p, s->pin_gather.p, gb + ib, cudaMemcpyHostToDevice, s->stream);
      if (e == cudaSuccess)
        e = launch_gather((const GatherDesc*)s->gather.p, (int)s->gdesc.size(),
                          (const int*)((char*)s->gather.p + gb), (double*)s->mats.p, s->stream);
      if (e != cudaSuccess) return fail(e, "gathering resident submatrices");
    }
  }
  // ---- queues
  size_t moff = 0, ioff = 0, noff = 0;
  char* pm = (char*)s->pin_meta.p;
  for (size_t g = 0; g < plans.size(); ++g) {
    Plan& P = plans[g];
    const int ni = (int)P.insts.size(), nit = (int)P.items.size();
    // shift item0 of every instance and the order entries to this group's slots
    std::memcpy(pm + moff, P.insts.data(), ni * sizeof(InstDesc));
    std::memcpy(pm + moff + ni * sizeof(InstDesc), P.items.data(), nit * sizeof(WorkItem));
    std::memcpy(pm + moff + ni * sizeof(InstDesc) + nit * sizeof(WorkItem), P.order.data(), nit * sizeof(int));
    gbs_session::Group G;
    ItemLaunch& L = G.L;
    char* dm = (char*)s->meta.p + moff;
    L.mats = (const double*)s->mats.p;
    L.insts = (const InstDesc*)dm;
    L.items = (const WorkItem*)(dm + ni * sizeof(InstDesc));
    L.order = (const int*)(dm + ni * sizeof(InstDesc) + nit * sizeof(WorkItem));
    L.n_items = nit;
    L.head = (int*)((char*)s->head.p + 64 * g);
    L.done = (int*)s->done.p + noff;
    L.part = (double*)s->part.p + 4 * ioff;
    L.paux = (double*)s->paux.p + ioff;
    L.pst = (int*)s->pst.p + ioff;
    L.out = (double*)s->out.p + 2 * noff;
    L.aux_out = (double*)s->aux.p + noff;
    L.st_out = (int*)s->st.p + noff;
    L.ws_doubles = P.ws_doubles;
    L.haf_smax = P.haf_smax;
    G.br = cover(P.need);
    // with a large shared workspace per warp (the hafnian families) the block size
    // that packs the most resident warps per SM (1, 2 or 4 warps: each block also
    // reserves shared memory of its own, so small blocks can lose a warp)
    const size_t smem_per_warp = (size_t)P.ws_doubles * sizeof(double);
    int warps = opt.warps;
    if (smem_per_warp >= 8192) {
      int best = 0;
      for (int w = 1; w <= 4; w <<= 1) {
        if ((size_t)w * smem_per_warp > 200 * 1024) break;
        const int resident = occ_any(G.br, L, w) * w;
        if (resident > best) { best = resident; warps = w; }
      }
      if (best == 0) warps = 1;
    }
    if (opt.per_size && !P.insts.empty()) {  // a per-size bucket: the tuned block size, if any
      const int tw = tuned_warps(ft_fn(P.insts[0].ft), ft_tier(P.insts[0].ft), P.insts[0].dim);
      if (tw > 0) warps = tw;
    }
    while (warps > 1 && (size_t)warps * smem_per_warp > 200 * 1024) warps >>= 1;
    const int bps = occ_any(G.br, L, warps);
    if (bps <= 0) return fail(cudaErrorInvalidConfiguration, "work item kernel does not fit on an SM");
    const long long want_blocks = (nit + warps - 1) / warps;
    G.grid = (int)std::min<long long>((long long)s->sms * bps, want_blocks);
    G.warps = warps;
    G.ni = ni;
    G.nit = nit;
    G.out_off = noff;
    G.req = greq[g];
    s->groups.push_back(std::move(G));
    moff += ((ni * sizeof(InstDesc) + nit * sizeof(WorkItem) + nit * sizeof(int)) + 255) & ~(size_t)255;
    ioff += nit;
    noff += ni;
  }
  if (moff > 0) {
    e = cudaMemcpyAsync(s->meta.p, pm, moff, cudaMemcpyHostToDevice, s->stream);
    if (e != cudaSuccess) return fail(e, "uploading the work queues");
  }
  s->plan_ninst = noff;
  s->plan_ready = true;
  return 0;
}

// Launch the prepared plan on `stream` (the session stream when null): reset the
// queue heads and completion counters, then one kernel per group.
// The launch sequence of the prepared plan: queue resets + one launch per group.
static cudaError_t plan_enqueue(gbs_session* s, cudaStream_t stream) {
  cudaError_t e = cudaSuccess;
  if (!s->groups.empty()) {
    e = cudaMemsetAsync(s->head.p, 0, 64 * s->groups.size(), stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(s->done.p, 0, s->plan_ninst * sizeof(int), stream);
  }
  for (auto& G : s->groups) {
    if (e != cudaSuccess) break;
    e = launch_any(G.br, G.L, G.grid, G.warps, stream);
    if (e != cudaSuccess)
      g_last_error = std::string("work item kernel (branch set ") + std::to_string(G.br) + ", grid " +
                     std::to_string(G.grid) + " x " + std::to_string(G.warps) + " warps, " +
                     std::to_string((size_t)G.warps * G.L.ws_doubles * sizeof(double)) + " B shared): " +
                     cudaGetErrorString(e);
  }
  return e;
}

// Run the prepared plan on `stream`.  From the second run of a plan on (the first
// run sets every kernel attribute), with graphs enabled, the sequence is captured
// once into a CUDA graph and replayed: one graph launch per run.
static int plan_launch(gbs_session* s, cudaStream_t stream, bool allow_graph = false) {
  if (!s->plan_ready) return fail(cudaErrorInvalidValue, "no prepared plan");
  if (!stream) stream = s->stream;
  cudaError_t e = cudaSuccess;
  long long items = 0;
  for (auto& G : s->groups) items += G.nit;
  const bool graph_now = allow_graph && s->use_graphs && !s->groups.empty() && s->plan_runs >= 1;
  if (graph_now && !s->graph) {
    cudaGraph_t g = nullptr;
    e = cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal);
    if (e == cudaSuccess) {
      const cudaError_t e1 = plan_enqueue(s, stream);
      e = cudaStreamEndCapture(stream, &g);
      if (e == cudaSuccess) e = e1;
    }
    if (e == cudaSuccess) e = cudaGraphInstantiate(&s->graph, g, 0);
    if (g) cudaGraphDestroy(g);
    if (e != cudaSuccess) {
      s->graph = nullptr;
      return fail(e, "capturing the plan's launch graph");
    }
  }
  cudaEventRecord(s->ev0, stream);
  g_last_error.clear();
  if (graph_now) e = cudaGraphLaunch(s->graph, stream);
  else e = plan_enqueue(s, stream);
  if (e != cudaSuccess) return fail(e, "launching the " + (g_last_error.empty() ? std::string("work item kernel") : g_last_error));
  cudaEventRecord(s->ev1, stream);
  s->plan_runs += 1;
  s->last_launches = (int)s->groups.size();
  s->last_items = items;
  return 0;
}

// Enqueue the device-to-host copies of the plan's results on `stream`.
static int plan_read_enqueue(gbs_session* s, cudaStream_t stream) {
  if (!stream) stream = s->stream;
  const size_t ni = s->plan_ninst;
  double* po = (double*)s->pin_out.p;
  double* pa = po + 2 * ni;
  int* ps = (int*)(pa + ni);
  cudaError_t e = cudaSuccess;
  if (ni > 0) {
    e = cudaMemcpyAsync(po, s->out.p, ni * 2 * sizeof(double), cudaMemcpyDeviceToHost, stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(pa, s->aux.p, ni * sizeof(double), cudaMemcpyDeviceToHost, stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(ps, s->st.p, ni * sizeof(int), cudaMemcpyDeviceToHost, stream);
  }
  return e == cudaSuccess ? 0 : fail(e, "reading results back");
}

// Scatter the (already copied) results to request order.
static void plan_collect(gbs_session* s, double* out, double* aux, int* st) {
  const size_t ni = s->plan_ninst;
  double* po = (double*)s->pin_out.p;
  double* pa = po + 2 * ni;
  int* ps = (int*)(pa + ni);
  for (const auto& G : s->groups)
    for (int k = 0; k < G.ni; ++k) {
      const int i = G.req[k];
      out[2 * i] = po[2 * (G.out_off + k)];
      out[2 * i + 1] = po[2 * (G.out_off + k) + 1];
      if (aux) aux[i] = pa[G.out_off + k];
      if (st) st[i] = ps[G.out_off + k];
    }
  for (int i = 0; i < s->plan_B; ++i) {
    if (!s->plan_trivial[i]) continue;
    const cplx t = s->plan_tval[i];
    out[2 * i] = t.re;
    out[2 * i + 1] = t.im;
    // exact values: bound 0 for the certified tiers, |value| as the indicator sum
    if (aux) aux[i] = tier_certified(s->plan_tier[i]) ? 0.0 : std::hypot(t.re, t.im);
    if (st) st[i] = kStOk;
  }
}

// Device-resident read: scatter the plan's results into a device block laid out as
// [B complex values][B doubles aux][B int32 status] (request order), on `stream`.
// `remap` (optional) sends request i of this plan to index remap[i] of the block;
// write_aux = false keeps the block's aux entries.
static int plan_scatter(gbs_session* s, cudaStream_t stream, double* block, int B_block,
                        const std::vector<int>* remap, bool write_aux) {
  if (!stream) stream = s->stream;
  const int ni = (int)s->plan_ninst;
  std::vector<int> tidx;
  std::vector<double> tval;
  for (int i = 0; i < s->plan_B; ++i) {
    if (!s->plan_trivial[i]) continue;
    const cplx t = s->plan_tval[i];
    tidx.push_back(remap ? (*remap)[i] : i);
    tval.push_back(t.re);
    tval.push_back(t.im);
    tval.push_back(tier_certified(s->plan_tier[i]) ? 0.0 : std::hypot(t.re, t.im));
  }
  const int nt = (int)tidx.size();
  if (ni + nt == 0) return 0;
  const size_t ints = ((size_t)ni + nt + 1) & ~(size_t)1;  // 8-byte boundary before the doubles
  const size_t bytes = ints * sizeof(int) + tval.size() * sizeof(double);
  cudaError_t e = cudaStreamSynchronize(stream);  // the pinned staging buffer is reused
  if (e == cudaSuccess) e = grow_pin(s->pin_rmap, bytes);
  if (e == cudaSuccess) e = grow_dev(s->rmap, bytes, &s->reallocs);
  if (e != cudaSuccess) return fail(e, "staging the resident result map");
  int* hm = (int*)s->pin_rmap.p;
  for (const auto& G : s->groups)
    for (int k = 0; k < G.ni; ++k) {
      const int i = G.req[k];
      hm[G.out_off + k] = remap ? (*remap)[i] : i;
    }
  for (int t = 0; t < nt; ++t) hm[ni + t] = tidx[t];
  double* hv = (double*)(hm + ints);
  for (size_t t = 0; t < tval.size(); ++t) hv[t] = tval[t];
  e = cudaMemcpyAsync(s->rmap.p, s->pin_rmap.p, bytes, cudaMemcpyHostToDevice, stream);
  if (e != cudaSuccess) return fail(e, "uploading the resident result map");
  ScatterArgs a{};
  a.out = (const double*)s->out.p;
  a.aux = (const double*)s->aux.p;
  a.st = (const int*)s->st.p;
  a.map = (const int*)s->rmap.p;
  a.ni = ni;
  a.tidx = (const int*)s->rmap.p + ni;
  a.tval = (const double*)((const int*)s->rmap.p + ints);
  a.ntriv = nt;
  a.dval = block;
  a.daux = block + 2 * (size_t)B_block;
  a.dst = (int*)(block + 3 * (size_t)B_block);
  a.write_aux = write_aux ? 1 : 0;
  e = launch_scatter(a, stream);
  return e == cudaSuccess ? 0 : fail(e, "scattering the resident results");
}

// Bytes of a resident result block of B requests.
static size_t resident_bytes(int B) { return (size_t)B * (3 * sizeof(double) + sizeof(int)); }

// Copy the plan's results back (synchronous) and scatter them to request order.
static int plan_read(gbs_session* s, cudaStream_t stream, double* out, double* aux, int* st) {
  if (!stream) stream = s->stream;
  int rc = plan_read_enqueue(s, stream);
  if (rc) return rc;
  cudaError_t e = cudaStreamSynchronize(stream);
  if (e != cudaSuccess) return fail(e, "evaluating the batch");
  float ms = 0.f;
  if (!s->groups.empty()) cudaEventElapsedTime(&ms, s->ev0, s->ev1);
  s->last_kernel_ms = ms;
  plan_collect(s, out, aux, st);
  return 0;
}

static int run_batch(gbs_session* s, const std::vector<Req>& reqs, double* out, double* aux, int* st,
                     const RunOpts& opt) {
  if (reqs.empty()) return 0;
  int rc = plan_build(s, reqs, opt);
  if (rc == 0) rc = plan_launch(s, nullptr);
  if (rc == 0) rc = plan_read(s, nullptr, out, aux, st);
  return rc;
}

// ------------------------------------------------------------------ process-wide default session
static std::mutex g_default_mu;
static gbs_session* g_default = nullptr;

static int session_open(gbs_session** out) {
  gbs_session* s = new gbs_session();
  cudaError_t e = cudaGetDevice(&s->device);
  if (e == cudaSuccess) e = cudaDeviceGetAttribute(&s->sms, cudaDevAttrMultiProcessorCount, s->device);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaEventCreate(&s->ev0);
  if (e == cudaSuccess) e = cudaEventCreate(&s->ev1);
  if (e != cudaSuccess) {
    delete s;
    *out = nullptr;
    return fail(e, "opening a session");
  }
  *out = s;
  return 0;
}

static void session_free(gbs_session* s) {
  if (!s) return;
  if (s->stream) cudaStreamSynchronize(s->stream);
  drop_graph(s);
  for (DevBuf* b : {&s->mats, &s->meta, &s->part, &s->paux, &s->pst, &s->done, &s->head, &s->out, &s->aux, &s->st,
                    &s->gather})
    if (b->p) cudaFree(b->p);
  for (PinBuf* b : {&s->pin_in, &s->pin_meta, &s->pin_out, &s->pin_gather})
    if (b->p) cudaFreeHost(b->p);
  if (s->ev0) cudaEventDestroy(s->ev0);
  if (s->ev1) cudaEventDestroy(s->ev1);
  if (s->stream) cudaStreamDestroy(s->stream);
  delete s;
}

static int with_default(gbs_session** s) {
  std::lock_guard<std::mutex> lk(g_default_mu);
  if (!g_default) {
    int rc = session_open(&g_default);
    if (rc) return rc;
  }
  *s = g_default;
  return 0;
}

// Uniform (B, d, d) batch through a session.
static int uniform(gbs_session* s, int fn, int tier, const double* m, int dim, int b, double* o, double* aux,
                   int* st) {
  if (b <= 0) return 0;
  if (!m || !o) return fail(cudaErrorInvalidValue, "null buffer");
  std::vector<Req> reqs(b);
  const size_t stride = 2ull * dim * dim;
  for (int i = 0; i < b; ++i) reqs[i] = Req{fn, tier, dim, m + i * stride};
  std::lock_guard<std::mutex> lk(s->mu);
  RunOpts opt;
  return run_batch(s, reqs, o, aux, st, opt);
}

// Status -> value convention of the reference: off-domain / uncertifiable -> NaN.
static void apply_status(int b, double* o, const int* st) {
  for (int i = 0; i < b; ++i)
    if (st[i] != kStOk) { o[2 * i] = NAN; o[2 * i + 1] = NAN; }
}

static int one_shot(int fn, int tier, const double* m, int dim, int b, double* o, double* aux) {
  gbs_session* s;
  int rc = with_default(&s);
  if (rc) return rc;
  std::vector<int> st(std::max(b, 0));
  rc = uniform(s, fn, tier, m, dim, b, o, aux, st.data());
  if (rc == 0) apply_status(b, o, st.data());
  return rc;
}

// auto tier: fp64 + indicator, then the elements with kappa >= threshold rerun in
// double-double on the device.  tier_out: 0 = fp64 kept, 1 = dd rerun.
static int auto_batch(gbs_session* s, const std::vector<Req>& reqs, double kappa_max, double* out, double* kappa,
                      int* tier_out, int* st) {
  const int B = (int)reqs.size();
  std::vector<Req> kreq = reqs;
  for (Req& r : kreq) r.tier = kTierKappa;
  std::vector<double> absn(B);
  RunOpts opt;
  int rc = run_batch(s, kreq, out, absn.data(), st, opt);
  if (rc) return rc;
  std::vector<Req> rerun;
  std::vector<int> idx;
  for (int i = 0; i < B; ++i) {
    const double mag = std::max(std::hypot(out[2 * i], out[2 * i + 1]), 1e-300);
    const double k = absn[i] / mag;
    if (kappa) kappa[i] = k;
    tier_out[i] = 0;
    if (st[i] == kStOk && !(k < kappa_max)) {
      Req r = reqs[i];
      r.tier = kTierDD;
      rerun.push_back(r);
      idx.push_back(i);
    }
  }
  if (!rerun.empty()) {
    std::vector<double> o2(2 * rerun.size());
    std::vector<int> s2(rerun.size());
    rc = run_batch(s, rerun, o2.data(), nullptr, s2.data(), opt);
    if (rc) return rc;
    for (size_t j = 0; j < idx.size(); ++j) {
      out[2 * idx[j]] = o2[2 * j];
      out[2 * idx[j] + 1] = o2[2 * j + 1];
      st[idx[j]] = s2[j];
      tier_out[idx[j]] = 1;
    }
  }
  return 0;
}

// Grow a session's plan buffers to hold `mat_bytes` of matrices, `items` work items
// and `insts` instances up front (the serving slots: a batch within the admission
// budget then never reallocates -- a device free or a pinned allocation would
// synchronise the GPU under every slot).
static int session_reserve(gbs_session* s, size_t mat_bytes, size_t items, size_t insts) {
  items = std::max<size_t>(items, 1);
  insts = std::max<size_t>(insts, 1);
  const size_t meta = insts * sizeof(InstDesc) + items * (sizeof(WorkItem) + sizeof(int)) + 1024;
  cudaError_t e = grow_pin(s->pin_in, std::max<size_t>(mat_bytes, 16));
  if (e == cudaSuccess) e = grow_dev(s->mats, std::max<size_t>(mat_bytes, 16), &s->reallocs);
  if (e == cudaSuccess) e = grow_pin(s->pin_meta, meta);
  if (e == cudaSuccess) e = grow_dev(s->meta, meta, &s->reallocs);
  if (e == cudaSuccess) e = grow_dev(s->part, items * 4 * sizeof(double), &s->reallocs);
  if (e == cudaSuccess) e = grow_dev(s->paux, items * sizeof(double), &s->reallocs);
  if (e == cudaSuccess) e = grow_dev(s->pst, items * sizeof(int), &s->reallocs);
  if (e == cudaSuccess) e = grow_dev(s->done, insts * sizeof(int), &s->reallocs);
  if (e == cudaSuccess) e = grow_dev(s->head, 64 * 8, &s->reallocs);
  if (e == cudaSuccess) e = grow_dev(s->out, insts * 2 * sizeof(double), &s->reallocs);
  if (e == cudaSuccess) e = grow_dev(s->aux, insts * sizeof(double), &s->reallocs);
  if (e == cudaSuccess) e = grow_dev(s->st, insts * sizeof(int), &s->reallocs);
  if (e == cudaSuccess) e = grow_pin(s->pin_out, insts * (3 * sizeof(double) + sizeof(int)));
  return e == cudaSuccess ? 0 : fail(e, "reserving the session buffers");
}

// Device-resident evaluation of `reqs` into `block` (resident_bytes(B), request
// order).  tier_mode >= 0: the requests' own tiers; kResidentAuto: fp64 + indicator,
// the elements with kappa >= kappa_max rerun in double-double and scattered over
// their fp64 values on the device; aux then holds kappa.  Only the kappa decision
// reads back to the host (values and sums), as the host auto tier does.
constexpr int kResidentAuto = -1;
static int resident_run(gbs_session* s, std::vector<Req> reqs, int tier_mode, double kappa_max, double* block) {
  const int B = (int)reqs.size();
  if (B == 0) return 0;
  RunOpts opt;
  auto finish = [&]() -> int {
    cudaError_t e = cudaStreamSynchronize(s->stream);
    if (e != cudaSuccess) return fail(e, "evaluating the batch");
    float ms = 0.f;
    if (!s->groups.empty()) cudaEventElapsedTime(&ms, s->ev0, s->ev1);
    s->last_kernel_ms = ms;
    return 0;
  };
  if (tier_mode == kResidentAuto)
    for (Req& r : reqs) r.tier = kTierKappa;
  int rc = plan_build(s, reqs, opt);
  if (rc == 0) rc = plan_launch(s, nullptr);
  if (rc == 0) rc = plan_scatter(s, nullptr, block, B, nullptr, true);
  if (rc == 0) rc = finish();
  if (rc || tier_mode != kResidentAuto) return rc;
  std::vector<double> val(2 * (size_t)B), absn(B);
  std::vector<int> st(B);
  cudaError_t e = cudaMemcpy(val.data(), block, val.size() * sizeof(double), cudaMemcpyDeviceToHost);
  if (e == cudaSuccess) e = cudaMemcpy(absn.data(), block + 2 * (size_t)B, B * sizeof(double), cudaMemcpyDeviceToHost);
  if (e == cudaSuccess) e = cudaMemcpy(st.data(), block + 3 * (size_t)B, B * sizeof(int), cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) return fail(e, "reading the indicator sums");
  std::vector<Req> rerun;
  std::vector<int> idx;
  std::vector<double> kap(B);
  for (int i = 0; i < B; ++i) {
    const double mag = std::max(std::hypot(val[2 * i], val[2 * i + 1]), 1e-300);
    kap[i] = absn[i] / mag;
    if (st[i] == kStOk && !(kap[i] < kappa_max)) {
      Req r = reqs[i];
      r.tier = kTierDD;
      rerun.push_back(r);
      idx.push_back(i);
    }
  }
  e = cudaMemcpy(block + 2 * (size_t)B, kap.data(), B * sizeof(double), cudaMemcpyHostToDevice);
  if (e != cudaSuccess) return fail(e, "writing kappa");
  if (rerun.empty()) return 0;
  rc = plan_build(s, rerun, opt);
  if (rc == 0) rc = plan_launch(s, nullptr);
  if (rc == 0) rc = plan_scatter(s, nullptr, block, B, &idx, false);
  if (rc == 0) rc = finish();
  return rc;
}

// A fresh resident block for B requests, evaluated; on failure nothing is kept.
static int resident_alloc_run(gbs_session* s, const std::vector<Req>& reqs, int tier_mode, double** d_block) {
  *d_block = nullptr;
  const int B = (int)reqs.size();
  if (B == 0) return 0;
  for (const Req& r : reqs)
    if (tier_certified(r.tier)) {
      const size_t nn = 2ull * (size_t)r.dim * r.dim;
      for (size_t k = 0; k < nn; ++k)
        if (!std::isfinite(r.mat[k])) return fail(cudaErrorInvalidValue, "certified evaluation requires finite input");
    }
  double* d = nullptr;
  cudaError_t e = cudaMalloc(&d, resident_bytes(B));
  if (e != cudaSuccess) return fail(e, "allocating the resident result block");
  std::lock_guard<std::mutex> lk(s->mu);
  const int rc = resident_run(s, reqs, tier_mode, 1e8, d);
  if (rc) {
    cudaFree(d);
    return rc;
  }
  *d_block = d;
  return 0;
}

}  // namespace gbsb

// ====================================================================== C ABI
using namespace gbsb;

extern "C" {

const char* gbs_last_error(void) { return g_last_error.c_str(); }

int gbs_version(void) { return 100; }

// ---- one-shot uniform batches (core/host_api.cu:150-268) --------------------
int gbs_perm_host(const double* m, int n, int b, double* o) { return one_shot(kFnPerm, kTierFp64, m, n, b, o, nullptr); }
int gbs_perm_dd_host(const double* m, int n, int b, double* o) { return one_shot(kFnPerm, kTierDD, m, n, b, o, nullptr); }
int gbs_haf_host(const double* m, int N, int b, double* o) { return one_shot(kFnHaf, kTierFp64, m, N, b, o, nullptr); }
int gbs_haf_dd_host(const double* m, int N, int b, double* o) { return one_shot(kFnHaf, kTierDD, m, N, b, o, nullptr); }
int gbs_lhaf_host(const double* m, int N, int b, double* o) { return one_shot(kFnLhaf, kTierFp64, m, N, b, o, nullptr); }
int gbs_lhaf_dd_host(const double* m, int N, int b, double* o) { return one_shot(kFnLhaf, kTierDD, m, N, b, o, nullptr); }
int gbs_tor_host(const double* m, int n, int b, double* o) { return one_shot(kFnTor, kTierFp64, m, 2 * n, b, o, nullptr); }
int gbs_tor_dd_host(const double* m, int n, int b, double* o) { return one_shot(kFnTor, kTierDD, m, 2 * n, b, o, nullptr); }

int gbs_perm_kappa_host(const double* m, int n, int b, double* o, double* a) { return one_shot(kFnPerm, kTierKappa, m, n, b, o, a); }
int gbs_haf_kappa_host(const double* m, int N, int b, double* o, double* a) { return one_shot(kFnHaf, kTierKappa, m, N, b, o, a); }
int gbs_lhaf_kappa_host(const double* m, int N, int b, double* o, double* a) { return one_shot(kFnLhaf, kTierKappa, m, N, b, o, a); }
int gbs_tor_kappa_host(const double* m, int n, int b, double* o, double* a) { return one_shot(kFnTor, kTierKappa, m, 2 * n, b, o, a); }

// ---- certified tier: value + rigorous bound (core/host_api.cu:248-262) ---------
static int one_shot_cert(int fn, const double* m, int dim, int b, double* o, double* bound, int tier = kTierCert) {
  if (b > 0 && !bound) return fail(cudaErrorInvalidValue, "null bound buffer");
  for (size_t i = 0; i < 2ull * (size_t)dim * dim * (size_t)std::max(b, 0); ++i)
    if (!std::isfinite(m[i])) return fail(cudaErrorInvalidValue, "certified evaluation requires finite input");
  int rc = one_shot(fn, tier, m, dim, b, o, bound);
  if (rc == 0)
    for (int i = 0; i < b; ++i)
      if (std::isnan(o[2 * i])) bound[i] = INFINITY;
  return rc;
}
int gbs_perm_certified_host(const double* m, int n, int b, double* o, double* e) { return one_shot_cert(kFnPerm, m, n, b, o, e); }
int gbs_haf_certified_host(const double* m, int N, int b, double* o, double* e) { return one_shot_cert(kFnHaf, m, N, b, o, e); }
int gbs_lhaf_certified_host(const double* m, int N, int b, double* o, double* e) { return one_shot_cert(kFnLhaf, m, N, b, o, e); }
int gbs_tor_certified_host(const double* m, int n, int b, double* o, double* e) { return one_shot_cert(kFnTor, m, 2 * n, b, o, e); }
// certified double-double permanent and torontonian: double-word value (returned
// rounded to binary64) + rigorous bound, the rung above the binary64 certificate
int gbs_perm_dd_certified_host(const double* m, int n, int b, double* o, double* e) {
  return one_shot_cert(kFnPerm, m, n, b, o, e, kTierCertDD);
}
int gbs_haf_dd_certified_host(const double* m, int N, int b, double* o, double* e) {
  return one_shot_cert(kFnHaf, m, N, b, o, e, kTierCertDD);
}
int gbs_lhaf_dd_certified_host(const double* m, int N, int b, double* o, double* e) {
  return one_shot_cert(kFnLhaf, m, N, b, o, e, kTierCertDD);
}
int gbs_tor_dd_certified_host(const double* m, int n, int b, double* o, double* e) {
  return one_shot_cert(kFnTor, m, 2 * n, b, o, e, kTierCertDD);
}

// ---- single-large torontonian (core/host_api.cu:270-352) ---------------------
// Real (2n x 2n) O, n <= 32, evaluated as ONE instance split into at least 2^g
// prefix work items over the whole GPU.  Off the physical domain the value is NaN
// (and the bound +inf); the certified variant returns the a-posteriori bound.
static int tor_single(int tier, const double* O, int n, int g, double* out, double* bound) {
  if (!O || !out || (tier_certified(tier) && !bound)) return fail(cudaErrorInvalidValue, "null pointer");
  if (n < 0 || n > kTorSingleCapModes) return fail(cudaErrorInvalidValue, "single-large torontonian: n must be in [0, 32]");
  if (g < 0 || g > n) return fail(cudaErrorInvalidValue, "single-large torontonian: groups must be in [0, n]");
  const int dim = 2 * n;
  std::vector<double> c(2 * (size_t)dim * dim, 0.0);
  for (size_t i = 0; i < (size_t)dim * dim; ++i) {
    if (!std::isfinite(O[i])) return fail(cudaErrorInvalidValue, "single-large torontonian: non-finite input");
    c[2 * i] = O[i];
  }
  gbs_session* s;
  int rc = with_default(&s);
  if (rc) return rc;
  Req r{};
  r.fn = kFnTor;
  r.tier = tier;
  r.dim = dim;
  r.mat = c.data();
  r.single = 1;
  r.split = g;
  double o[2] = {0.0, 0.0}, aux = 0.0;
  int st = 0;
  RunOpts opt;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    rc = run_batch(s, std::vector<Req>{r}, o, &aux, &st, opt);
  }
  if (rc) return rc;
  const bool ok = st == kStOk && std::isfinite(o[0]);
  *out = ok ? o[0] : NAN;
  if (bound) *bound = ok ? aux : INFINITY;
  return 0;
}
int gbs_tor_recursive_single_host(const double* O, int n, int g, double* out) {
  return tor_single(kTierFp64, O, n, g, out, nullptr);
}
int gbs_tor_single_certified_host(const double* O, int n, int g, double* out, double* bound) {
  return tor_single(kTierCert, O, n, g, out, bound);
}
int gbs_tor_single_ddcertified_host(const double* O, int n, int g, double* out, double* bound) {
  return tor_single(kTierCertDD, O, n, g, out, bound);
}

// ---- auto tier on the device (gbskernels/__init__.py:272-297) ----------------
// func: 0 perm, 1 haf, 2 lhaf, 3 tor; dim = matrix side.  tier_out: 0 fp64, 1 dd.
int gbs_auto_host(int func, const double* m, int dim, int b, double kappa_max, double* o, double* kappa,
                  int* tier_out) {
  if (b <= 0) return 0;
  if (!m || !o || !tier_out) return fail(cudaErrorInvalidValue, "null buffer");
  gbs_session* s;
  int rc = with_default(&s);
  if (rc) return rc;
  std::vector<Req> reqs(b);
  const size_t stride = 2ull * dim * dim;
  for (int i = 0; i < b; ++i) reqs[i] = Req{func, kTierFp64, dim, m + i * stride};
  std::vector<int> st(b);
  std::lock_guard<std::mutex> lk(s->mu);
  rc = auto_batch(s, reqs, kappa_max, o, kappa, tier_out, st.data());
  if (rc == 0) apply_status(b, o, st.data());
  return rc;
}

// ---- certified tier with the proven rtol ladder (gbskernels/__init__.py:374-478) ----
// The binary64 certificate first; every element whose bound does not prove a
// relative error <= rtol (or is not finite) is re-evaluated by the certified
// double-double rung in one more launch.  tier_out[i]: 3 certified binary64,
// 4 certified double-double, -1 no rung certifies it.  rtol < 0: no ladder (the
// binary64 certificate as it is; -1 where it is not finite).  The reference's last
// rung (mpmath on the host) has no counterpart: a refused element stays refused.
static bool certificate_meets(double re, double im, double e, double rtol) {
  if (!(std::isfinite(re) && std::isfinite(im) && std::isfinite(e) && e >= 0.0)) return false;
  if (rtol < 0.0) return true;
  const double mag = std::hypot(re, im);
  if (mag == 0.0) return e == 0.0;
  return e / mag <= rtol;
}

int gbs_certified_ladder_host(int func, const double* m, int dim, int b, double rtol, double* o, double* bound,
                              int* tier_out) {
  if (b <= 0) return 0;
  if (!m || !o || !bound || !tier_out) return fail(cudaErrorInvalidValue, "null buffer");
  if (func < kFnPerm || func > kFnTor) return fail(cudaErrorInvalidValue, "unknown function code");
  if (func == kFnTor && (dim & 1)) return fail(cudaErrorInvalidValue, "torontonian: matrix side must be even");
  int rc = one_shot_cert(func, m, dim, b, o, bound, kTierCert);
  if (rc) return rc;
  const size_t nn = 2ull * (size_t)dim * dim;
  std::vector<int> redo;
  for (int i = 0; i < b; ++i) {
    const bool ok = certificate_meets(o[2 * i], o[2 * i + 1], bound[i], rtol);
    tier_out[i] = ok ? kTierCert : -1;
    bool real = true;  // the double-double torontonian is real-domain only
    if (func == kFnTor)
      for (size_t k = 1; k < nn && real; k += 2) real = m[i * nn + k] == 0.0;
    if (!ok && rtol >= 0.0 && real) redo.push_back(i);
  }
  if (redo.empty()) return 0;
  std::vector<double> sub(nn * redo.size()), o2(2 * redo.size()), b2(redo.size());
  for (size_t j = 0; j < redo.size(); ++j) std::memcpy(&sub[j * nn], m + redo[j] * nn, nn * sizeof(double));
  rc = one_shot_cert(func, sub.data(), dim, (int)redo.size(), o2.data(), b2.data(), kTierCertDD);
  if (rc) return rc;
  for (size_t j = 0; j < redo.size(); ++j) {
    if (!certificate_meets(o2[2 * j], o2[2 * j + 1], b2[j], rtol)) continue;
    const int i = redo[j];
    o[2 * i] = o2[2 * j];
    o[2 * i + 1] = o2[2 * j + 1];
    bound[i] = b2[j];
    tier_out[i] = kTierCertDD;
  }
  return 0;
}

// ---- sessions (core/host_api.cu:521-658) --------------------------------------
int gbs_session_open(gbs_session** out) {
  if (!out) return fail(cudaErrorInvalidValue, "null session pointer");
  return session_open(out);
}
int gbs_session_close(gbs_session* s) {
  session_free(s);
  return 0;
}
size_t gbs_session_reallocs(const gbs_session* s) { return s ? s->reallocs : 0; }

// func: 0 perm, 1 haf, 2 lhaf, 3 tor; prec: 0 fp64, 1 dd, 2 fp64 + sum|term| (aux).
int gbs_session_evaluate(gbs_session* s, int func, int prec, const double* h_mats, int dim, int batch,
                         double* h_out) {
  if (!s) return fail(cudaErrorInvalidValue, "null session");
  if (batch <= 0) return 0;
  std::vector<int> st(batch);
  int rc = uniform(s, func, prec, h_mats, dim, batch, h_out, nullptr, st.data());
  if (rc == 0) apply_status(batch, h_out, st.data());
  return rc;
}

// Device-resident output: evaluate, then scatter the (B,) complex results on the
// device into a fresh buffer owned by the caller (freed by gbs_dev_free); nothing
// of the result passes through the host.  prec: 0 fp64, 1 dd.
int gbs_session_evaluate_resident(gbs_session* s, int func, int prec, const double* h_mats, int dim, int batch,
                                  double** d_result) {
  if (!s || !d_result) return fail(cudaErrorInvalidValue, "null argument");
  *d_result = nullptr;
  if (batch <= 0) return 0;
  if (!h_mats) return fail(cudaErrorInvalidValue, "null buffer");
  if (prec != 0 && prec != 1) return fail(cudaErrorInvalidValue, "prec must be 0 (fp64) or 1 (dd)");
  std::vector<Req> reqs(batch);
  const size_t stride = 2ull * dim * dim;
  for (int i = 0; i < batch; ++i) reqs[i] = Req{func, prec, dim, h_mats + i * stride};
  return resident_alloc_run(s, reqs, prec, d_result);
}
// Every tier, resident: a block [B complex values][B doubles aux][B int32 status].
// tier: 0 fp64, 1 dd, 2 fp64 + sum|term| (aux), 3 certified (aux = bound),
// 4 certified double-double (perm, tor), -1 auto (aux = kappa; kappa >= 1e8 -> dd).
int gbs_session_evaluate_resident_tier(gbs_session* s, int func, int tier, const double* h_mats, int dim, int batch,
                                       double** d_block) {
  if (!s || !d_block) return fail(cudaErrorInvalidValue, "null argument");
  *d_block = nullptr;
  if (batch <= 0) return 0;
  if (!h_mats) return fail(cudaErrorInvalidValue, "null buffer");
  if (tier < -1 || tier > 4) return fail(cudaErrorInvalidValue, "unsupported precision tier");
  std::vector<Req> reqs(batch);
  const size_t stride = 2ull * dim * dim;
  for (int i = 0; i < batch; ++i) reqs[i] = Req{func, tier < 0 ? kTierFp64 : tier, dim, h_mats + i * stride};
  return resident_alloc_run(s, reqs, tier, d_block);
}
// Ragged / mixed batch, resident (the queue of gbs_queue_evaluate; results in
// request order in a block as above).
int gbs_queue_evaluate_resident(gbs_session* s, int B, const int* funcs, const int* tiers, const int* dims,
                                const long long* offsets, const double* mats, int mode, double** d_block) {
  if (!s || !d_block) return fail(cudaErrorInvalidValue, "null argument");
  *d_block = nullptr;
  if (B <= 0) return 0;
  if (!funcs || !tiers || !dims || !offsets || !mats) return fail(cudaErrorInvalidValue, "null buffer");
  std::vector<Req> reqs(B);
  for (int i = 0; i < B; ++i) reqs[i] = Req{funcs[i], tiers[i], dims[i], mats + 2 * offsets[i]};
  (void)mode;  // results are identical in either launch mode; the persistent queue is used
  return resident_alloc_run(s, reqs, 0, d_block);
}
// The device that owns device memory `d` (for DLPack export of resident results).
int gbs_dev_device(const void* d, int* device) {
  if (!d || !device) return fail(cudaErrorInvalidValue, "null argument");
  cudaPointerAttributes at{};
  const cudaError_t e = cudaPointerGetAttributes(&at, d);
  if (e != cudaSuccess) return fail(e, "querying a device pointer");
  *device = at.device;
  return 0;
}
int gbs_dev_copy_to_host(const void* d, void* h, size_t bytes) {
  if (bytes == 0) return 0;
  if (!d || !h) return fail(cudaErrorInvalidValue, "null buffer");
  return (int)cudaMemcpy(h, d, bytes, cudaMemcpyDeviceToHost);
}
int gbs_dev_to_host(const double* d, double* h, int n) {
  if (n <= 0) return 0;
  return (int)cudaMemcpy(h, d, (size_t)n * 2 * sizeof(double), cudaMemcpyDeviceToHost);
}
int gbs_dev_free(double* d) {
  cudaFree(d);
  return 0;
}

// ---- ragged / mixed batches ----------------------------------------------------
// B requests: funcs[i], tiers[i] (0 fp64, 1 dd, 2 fp64 + sum|term|), dims[i] (matrix
// side), offsets[i] (in complex elements) into the packed host buffer `mats`.
// mode: 0 = persistent mixed queue (one launch), 1 = plain per-size launches.
int gbs_queue_evaluate(gbs_session* s, int B, const int* funcs, const int* tiers, const int* dims,
                       const long long* offsets, const double* mats, int mode, double* out, double* aux,
                       int* status) {
  if (!s) return fail(cudaErrorInvalidValue, "null session");
  if (B <= 0) return 0;
  if (!funcs || !tiers || !dims || !offsets || !mats || !out) return fail(cudaErrorInvalidValue, "null buffer");
  std::vector<Req> reqs(B);
  for (int i = 0; i < B; ++i) reqs[i] = Req{funcs[i], tiers[i], dims[i], mats + 2 * offsets[i]};
  std::vector<int> st(B);
  RunOpts opt;
  opt.per_size = (mode == 1);
  std::lock_guard<std::mutex> lk(s->mu);
  int rc = run_batch(s, reqs, out, aux, st.data(), opt);
  if (rc) return rc;
  if (status) std::memcpy(status, st.data(), sizeof(int) * B);
  apply_status(B, out, st.data());
  return 0;
}

// As gbs_queue_evaluate, with one host pointer per matrix instead of one packed
// buffer: the matrices are copied once, straight into the session's pinned staging
// buffer, so a caller holding B separate arrays does not pack them first.
int gbs_queue_evaluate_ptrs(gbs_session* s, int B, const int* funcs, const int* tiers, const int* dims,
                            const double* const* mats, int mode, double* out, double* aux, int* status) {
  if (!s) return fail(cudaErrorInvalidValue, "null session");
  if (B <= 0) return 0;
  if (!funcs || !tiers || !dims || !mats || !out) return fail(cudaErrorInvalidValue, "null buffer");
  std::vector<Req> reqs(B);
  for (int i = 0; i < B; ++i) {
    if (!mats[i] && dims[i] > 0) return fail(cudaErrorInvalidValue, "null matrix pointer");
    reqs[i] = Req{funcs[i], tiers[i], dims[i], mats[i]};
  }
  std::vector<int> st(B);
  RunOpts opt;
  opt.per_size = (mode == 1);
  std::lock_guard<std::mutex> lk(s->mu);
  int rc = run_batch(s, reqs, out, aux, st.data(), opt);
  if (rc) return rc;
  if (status) std::memcpy(status, st.data(), sizeof(int) * B);
  apply_status(B, out, st.data());
  return 0;
}

// Ragged / mixed batch in the auto tier: every request's fp64 value with its
// indicator in one launch, then the requests with kappa >= kappa_max rerun in
// double-double in one more (gbskernels/__init__.py:272-297 per element, without
// the reference's per-size buckets).  tier_out[i]: 0 fp64 kept, 1 dd rerun.
int gbs_queue_evaluate_auto(gbs_session* s, int B, const int* funcs, const int* dims, const long long* offsets,
                            const double* mats, double kappa_max, double* out, double* kappa, int* tier_out,
                            int* status) {
  if (!s) return fail(cudaErrorInvalidValue, "null session");
  if (B <= 0) return 0;
  if (!funcs || !dims || !offsets || !mats || !out || !tier_out) return fail(cudaErrorInvalidValue, "null buffer");
  std::vector<Req> reqs(B);
  for (int i = 0; i < B; ++i) reqs[i] = Req{funcs[i], kTierFp64, dims[i], mats + 2 * offsets[i]};
  std::vector<int> st(B);
  std::lock_guard<std::mutex> lk(s->mu);
  const int rc = auto_batch(s, reqs, kappa_max, out, kappa, tier_out, st.data());
  if (rc) return rc;
  if (status) std::memcpy(status, st.data(), sizeof(int) * B);
  apply_status(B, out, st.data());
  return 0;
}

// Device-resident plan: upload + cut once (gbs_queue_prepare), launch many times
// (gbs_queue_run, on `stream` or the session stream when null), read back
// (gbs_queue_read).  Inputs stay in HBM between runs.
int gbs_queue_prepare(gbs_session* s, int B, const int* funcs, const int* tiers, const int* dims,
                      const long long* offsets, const double* mats, int mode) {
  if (!s) return fail(cudaErrorInvalidValue, "null session");
  if (B < 0 || (B > 0 && (!funcs || !tiers || !dims || !offsets || !mats)))
    return fail(cudaErrorInvalidValue, "null buffer");
  std::vector<Req> reqs(B);
  for (int i = 0; i < B; ++i) reqs[i] = Req{funcs[i], tiers[i], dims[i], mats + 2 * offsets[i]};
  RunOpts opt;
  opt.per_size = (mode == 1);
  std::lock_guard<std::mutex> lk(s->mu);
  int rc = plan_build(s, reqs, opt);
  if (rc == 0) {
    cudaError_t e = cudaStreamSynchronize(s->stream);
    if (e != cudaSuccess) rc = fail(e, "uploading the plan");
  }
  return rc;
}
int gbs_queue_run(gbs_session* s, void* stream) {
  if (!s) return fail(cudaErrorInvalidValue, "null session");
  std::lock_guard<std::mutex> lk(s->mu);
  return plan_launch(s, (cudaStream_t)stream, true);
}

// Autotuner hooks: split = log2 of the work per item (haf / lhaf: subsets per item;
// perm: Gray steps per lane; tor: prefix leaves per item, or subsets per lane in the
// double-double tier); warps = block size of per-size launches; -1 / 0 = default.
int gbs_set_split(int func, int tier, int dim, int split, int warps) {
  if (func < 0 || func > 3 || tier < 0 || tier > 4 || dim < 0 || dim >= kTuneDims || split < -1 || split > 40 ||
      warps < 0 || warps > 8)
    return fail(cudaErrorInvalidValue, "gbs_set_split: argument out of range");
  const int t = (tier == kTierDD || tier == kTierCertDD) ? 1 : 0;
  g_tune_split[func][t][dim].store(split + 1);
  g_tune_warps[func][t][dim].store(warps);
  return 0;
}
int gbs_get_split(int func, int tier, int dim, int* split, int* warps) {
  if (func < 0 || func > 3 || tier < 0 || tier > 4 || dim < 0 || dim >= kTuneDims)
    return fail(cudaErrorInvalidValue, "gbs_get_split: argument out of range");
  if (split) *split = tuned_split(func, tier, dim);
  if (warps) *warps = tuned_warps(func, tier, dim);
  return 0;
}

int gbs_session_set_graphs(gbs_session* s, int enable) {
  if (!s) return fail(cudaErrorInvalidValue, "null session");
  std::lock_guard<std::mutex> lk(s->mu);
  s->use_graphs = enable != 0;
  if (!s->use_graphs) drop_graph(s);
  return 0;
}
int gbs_queue_read(gbs_session* s, void* stream, double* out, double* aux, int* status) {
  if (!s || !out) return fail(cudaErrorInvalidValue, "null argument");
  std::lock_guard<std::mutex> lk(s->mu);
  std::vector<int> st(std::max(s->plan_B, 1));
  int rc = plan_read(s, (cudaStream_t)stream, out, aux, st.data());
  if (rc) return rc;
  if (status) std::memcpy(status, st.data(), sizeof(int) * s->plan_B);
  apply_status(s->plan_B, out, st.data());
  return 0;
}

// Launch statistics of the session's last evaluation.
int gbs_session_last_stats(const gbs_session* s, double* kernel_ms, int* launches, long long* items) {
  if (!s) return fail(cudaErrorInvalidValue, "null session");
  if (kernel_ms) *kernel_ms = s->last_kernel_ms;
  if (launches) *launches = s->last_launches;
  if (items) *items = s->last_items;
  return 0;
}

}  // extern "C"

// ====================================================================== serving loop
// Continuous batching for chain-rule sampler queries (new; the reference serves no
// requests -- its resident sampler session, core/sampler_session.cu:68-128, runs a
// fixed chain).  A scheduler thread owns `slots` sessions (one stream each):
//   1. a finished slot (its completion event has fired) delivers its results --
//      an "auto" request whose indicator reaches kappa_max goes back to the front of
//      the queue as a double-double request with the same ticket;
//   2. a free slot admits the oldest pending requests up to the workspace budget
//      (matrix bytes + per-item partials) and launches them as ONE persistent queue;
//   3. with nothing to do it waits on the submission condition variable (bounded).
// Requests that arrive while batches are on the GPU join the next free slot, so
// up to `slots` batches overlap on the device.  A value never depends on its batch
// (work items are a function of the request alone).
#include <chrono>
#include <condition_variable>
#include <deque>
#include <thread>
#include <unordered_map>

namespace gbsb {

static double now_s() {
  return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

struct SrvReq {
  long long ticket = 0;
  int fn = 0, tier = 0, dim = 0;
  bool is_auto = false;
  std::vector<double> mat;
  int state = -1;
  std::vector<int> idx;
  bool use_gamma = false;
  double t_submit = 0.0;
};
struct SrvRes {
  double re = 0, im = 0, aux = 0;
  int status = 0, tier_used = 0;
  double t_submit = 0, t_done = 0;
  bool done = false;
};
struct SrvState {
  double* dA = nullptr;
  double* dG = nullptr;
  int M = 0;
  int real = 0;
};
struct Slot {
  gbs_session* s = nullptr;
  bool busy = false;
  std::vector<SrvReq> batch;
  cudaEvent_t done = nullptr;
};

}  // namespace gbsb

struct gbs_server {
  std::vector<gbsb::Slot> slots;
  std::vector<gbsb::SrvState> states;
  std::deque<gbsb::SrvReq> pending;
  std::unordered_map<long long, gbsb::SrvRes> results;
  std::mutex mu;
  std::condition_variable cv;
  std::thread worker;
  bool stop = false;
  int error = 0;
  std::string error_msg;
  long long next_ticket = 1;
  size_t budget = 0;
  int max_batch = 0;
  double kappa_max = 1e8;
  long long batches = 0, completed = 0, in_flight = 0;
  int device = 0;
};

namespace gbsb {

static size_t req_bytes(const SrvReq& r) {
  const size_t d = (size_t)r.dim + 1;
  size_t items = 1;
  if (r.fn == kFnHaf || r.fn == kFnLhaf) items = (size_t)1 << std::max(0, (int)(d / 2) - 7);
  return d * d * 16 + items * 48 + 256;
}

static int srv_launch(gbs_server* sv, Slot& sl) {
  std::vector<Req> reqs(sl.batch.size());
  for (size_t i = 0; i < sl.batch.size(); ++i) {
    const SrvReq& q = sl.batch[i];
    Req r{q.fn, q.tier, q.dim, q.mat.empty() ? nullptr : q.mat.data()};
    if (q.state >= 0) {
      const SrvState& S = sv->states[q.state];
      r.state = S.dA;
      r.gamma = q.use_gamma ? S.dG : nullptr;
      r.idx = q.idx.data();
      r.M = S.M;
      r.state_real = S.real;
    }
    reqs[i] = r;
  }
  RunOpts opt;
  int rc = plan_build(sl.s, reqs, opt);
  if (rc == 0) rc = plan_launch(sl.s, nullptr);
  if (rc == 0) rc = plan_read_enqueue(sl.s, nullptr);
  if (rc == 0) {
    cudaError_t e = cudaEventRecord(sl.done, sl.s->stream);
    if (e != cudaSuccess) rc = fail(e, "recording a completion event");
  }
  return rc;
}

static void srv_loop(gbs_server* sv) {
  cudaSetDevice(sv->device);
  std::unique_lock<std::mutex> lk(sv->mu);
  for (;;) {
    bool progressed = false;
    // 1. completions
    for (Slot& sl : sv->slots) {
      if (!sl.busy) continue;
      cudaError_t q = cudaEventQuery(sl.done);
      if (q == cudaErrorNotReady) continue;
      const size_t B = sl.batch.size();
      std::vector<double> out(2 * B), aux(B);
      std::vector<int> st(B);
      if (q != cudaSuccess) {
        sv->error = (int)q;
        sv->error_msg = "serving batch failed";
        for (size_t i = 0; i < B; ++i) st[i] = kStTimeout;
      } else {
        plan_collect(sl.s, out.data(), aux.data(), st.data());
      }
      const double t = now_s();
      for (size_t i = 0; i < B; ++i) {
        SrvReq& r = sl.batch[i];
        if (r.is_auto && r.tier == kTierKappa && st[i] == kStOk) {
          const double mag = std::max(std::hypot(out[2 * i], out[2 * i + 1]), 1e-300);
          if (!(aux[i] / mag < sv->kappa_max)) {
            SrvReq again = r;
            again.tier = kTierDD;
            sv->pending.push_front(std::move(again));
            sv->results[r.ticket].aux = aux[i] / mag;
            continue;
          }
        }
        SrvRes& res = sv->results[r.ticket];
        res.re = out[2 * i];
        res.im = out[2 * i + 1];
        if (st[i] != kStOk) { res.re = NAN; res.im = NAN; }
        if (r.is_auto) {
          if (r.tier == kTierKappa) res.aux = aux[i] / std::max(std::hypot(res.re, res.im), 1e-300);
          res.tier_used = r.tier == kTierDD ? 1 : 0;
        } else {
          res.aux = (r.tier == kTierCert && st[i] != kStOk) ? INFINITY : aux[i];
          res.tier_used = r.tier;
        }
        res.status = st[i];
        res.t_done = t;
        res.done = true;
        ++sv->completed;
      }
      sv->in_flight -= (long long)B;
      sl.batch.clear();
      sl.busy = false;
      progressed = true;
    }
    // 2. admission
    for (Slot& sl : sv->slots) {
      if (sl.busy || sv->pending.empty()) continue;
      size_t bytes = 0;
      while (!sv->pending.empty() && (int)sl.batch.size() < sv->max_batch) {
        const size_t b = req_bytes(sv->pending.front());
        if (!sl.batch.empty() && bytes + b > sv->budget) break;
        bytes += b;
        sl.batch.push_back(std::move(sv->pending.front()));
        sv->pending.pop_front();
      }
      sv->in_flight += (long long)sl.batch.size();
      lk.unlock();
      int rc = srv_launch(sv, sl);
      lk.lock();
      if (rc) {
        sv->error = rc;
        sv->error_msg = g_last_error;
        for (SrvReq& r : sl.batch) {
          SrvRes& res = sv->results[r.ticket];
          res.re = res.im = NAN;
          res.status = kStTimeout;
          res.done = true;
          res.t_done = now_s();
          ++sv->completed;
        }
        sv->in_flight -= (long long)sl.batch.size();
        sl.batch.clear();
      } else {
        sl.busy = true;
        ++sv->batches;
      }
      progressed = true;
    }
    bool any_busy = false;
    for (Slot& sl : sv->slots) any_busy |= sl.busy;
    if (sv->stop && sv->pending.empty() && !any_busy) break;
    if (!progressed) {
      if (any_busy) {
        // poll the completion events at a fine granularity without holding the lock
        lk.unlock();
        std::this_thread::sleep_for(std::chrono::microseconds(20));
        lk.lock();
      } else {
        sv->cv.wait_for(lk, std::chrono::milliseconds(2));
      }
    }
  }
}

}  // namespace gbsb

extern "C" {

// Open a server with `n_slots` concurrent batches, a per-batch workspace budget in
// bytes (admission control) and a per-batch request cap.
int gbs_server_open(int n_slots, long long budget_bytes, int max_batch, gbs_server** out) {
  if (!out || n_slots < 1 || n_slots > 64) return fail(cudaErrorInvalidValue, "bad server arguments");
  gbs_server* sv = new gbs_server();
  cudaGetDevice(&sv->device);
  sv->budget = budget_bytes > 0 ? (size_t)budget_bytes : ((size_t)256 << 20);
  sv->max_batch = max_batch > 0 ? max_batch : 4096;
  sv->slots.resize(n_slots);
  // per slot, buffers for a batch at the admission budget (req_bytes charges d^2 x 16
  // bytes of matrix and 48 bytes per work item), so serving never reallocates
  // (at most 256 MB of matrices per slot up front; a larger budget grows on demand)
  const size_t rbytes = std::min<size_t>(sv->budget, (size_t)256 << 20);
  const size_t insts = std::min<size_t>((size_t)sv->max_batch, rbytes / 256 + 1);
  for (Slot& sl : sv->slots) {
    int rc = session_open(&sl.s);
    if (rc == 0) rc = session_reserve(sl.s, rbytes, rbytes / 48 + 1, insts);
    cudaError_t e = rc == 0 ? cudaEventCreateWithFlags(&sl.done, cudaEventDisableTiming) : cudaErrorUnknown;
    if (rc || e != cudaSuccess) {
      for (Slot& t : sv->slots) {
        if (t.s) session_free(t.s);
        if (t.done) cudaEventDestroy(t.done);
      }
      delete sv;
      return fail(rc ? rc : (int)e, "opening server slots");
    }
  }
  sv->worker = std::thread(srv_loop, sv);
  *out = sv;
  return 0;
}

// Drain every pending request, stop the scheduler and free the slots.
int gbs_server_close(gbs_server* sv) {
  if (!sv) return 0;
  {
    std::lock_guard<std::mutex> lk(sv->mu);
    sv->stop = true;
  }
  sv->cv.notify_all();
  if (sv->worker.joinable()) sv->worker.join();
  for (Slot& sl : sv->slots) {
    if (sl.s) session_free(sl.s);
    if (sl.done) cudaEventDestroy(sl.done);
  }
  for (SrvState& st : sv->states) {
    if (st.dA) cudaFree(st.dA);
    if (st.dG) cudaFree(st.dG);
  }
  delete sv;
  return 0;
}

// Upload a resident state: an M x M complex matrix (the GBS kernel A, or O in
// xxpp for torontonians) and optional M loop weights.  Returns its id.
int gbs_server_add_state(gbs_server* sv, const double* A, const double* gamma, int M, int* state_id) {
  if (!sv || !A || M <= 0 || !state_id) return fail(cudaErrorInvalidValue, "bad state arguments");
  SrvState S;
  S.M = M;
  S.real = 1;
  for (size_t i = 0; i < (size_t)M * M; ++i)
    if (A[2 * i + 1] != 0.0) { S.real = 0; break; }
  cudaError_t e = cudaMalloc(&S.dA, (size_t)M * M * 16);
  if (e == cudaSuccess) e = cudaMemcpy(S.dA, A, (size_t)M * M * 16, cudaMemcpyHostToDevice);
  if (e == cudaSuccess && gamma) {
    e = cudaMalloc(&S.dG, (size_t)M * 16);
    if (e == cudaSuccess) e = cudaMemcpy(S.dG, gamma, (size_t)M * 16, cudaMemcpyHostToDevice);
  }
  if (e != cudaSuccess) {
    if (S.dA) cudaFree(S.dA);
    if (S.dG) cudaFree(S.dG);
    return fail(e, "uploading a resident state");
  }
  std::lock_guard<std::mutex> lk(sv->mu);
  sv->states.push_back(S);
  *state_id = (int)sv->states.size() - 1;
  return 0;
}

static int srv_submit(gbs_server* sv, gbsb::SrvReq&& r, long long* ticket) {
  if (r.tier < 0 || r.tier > 3) return fail(cudaErrorInvalidValue, "tier must be 0 fp64, 1 dd, 2 auto, 3 certified");
  if (r.tier == 2) { r.is_auto = true; r.tier = kTierKappa; }
  r.t_submit = now_s();
  {
    std::lock_guard<std::mutex> lk(sv->mu);
    if (sv->stop) return fail(cudaErrorInvalidValue, "server is closing");
    r.ticket = sv->next_ticket++;
    SrvRes& res = sv->results[r.ticket];
    res.t_submit = r.t_submit;
    *ticket = r.ticket;
    sv->pending.push_back(std::move(r));
  }
  sv->cv.notify_one();
  return 0;
}

// Submit one request with an explicit matrix (dim x dim complex; tor: 2n x 2n).
// tier: 0 fp64, 1 dd, 2 auto (fp64 + indicator, double-double rerun), 3 certified.
int gbs_server_submit(gbs_server* sv, int func, int tier, int dim, const double* mat, long long* ticket) {
  if (!sv || !ticket || dim < 0 || (dim > 0 && !mat)) return fail(cudaErrorInvalidValue, "bad request");
  gbsb::SrvReq r;
  r.fn = func;
  r.tier = tier;
  r.dim = dim;
  r.mat.assign(mat, mat + 2 * (size_t)dim * dim);
  return srv_submit(sv, std::move(r), ticket);
}

// Submit one request on a resident state: the matrix is state[idx][:, idx]
// (use_gamma: the state's loop weights on the diagonal), gathered on the device.
int gbs_server_submit_state(gbs_server* sv, int func, int tier, int state, int n_idx, const int* idx, int use_gamma,
                            long long* ticket) {
  if (!sv || !ticket || n_idx < 0 || (n_idx > 0 && !idx)) return fail(cudaErrorInvalidValue, "bad request");
  {
    std::lock_guard<std::mutex> lk(sv->mu);
    if (state < 0 || state >= (int)sv->states.size()) return fail(cudaErrorInvalidValue, "unknown state");
    for (int i = 0; i < n_idx; ++i)
      if (idx[i] < 0 || idx[i] >= sv->states[state].M) return fail(cudaErrorInvalidValue, "index outside the state");
    if (use_gamma && !sv->states[state].dG) return fail(cudaErrorInvalidValue, "state has no loop weights");
  }
  gbsb::SrvReq r;
  r.fn = func;
  r.tier = tier;
  r.dim = n_idx;
  r.state = state;
  r.idx.assign(idx, idx + n_idx);
  r.use_gamma = use_gamma != 0;
  return srv_submit(sv, std::move(r), ticket);
}

// Non-blocking poll.  When done: out = value (complex), aux = kappa (auto) or bound
// (certified), tier_used (0 fp64, 1 dd, 3 certified), latency_s = completion -
// submission; the result is then released.
int gbs_server_poll(gbs_server* sv, long long ticket, int* done, double* out, double* aux, int* status,
                    int* tier_used, double* latency_s) {
  if (!sv || !done) return fail(cudaErrorInvalidValue, "null argument");
  std::lock_guard<std::mutex> lk(sv->mu);
  auto it = sv->results.find(ticket);
  if (it == sv->results.end()) return fail(cudaErrorInvalidValue, "unknown ticket");
  *done = it->second.done ? 1 : 0;
  if (!it->second.done) return 0;
  const SrvRes& r = it->second;
  if (out) { out[0] = r.re; out[1] = r.im; }
  if (aux) *aux = r.aux;
  if (status) *status = r.status;
  if (tier_used) *tier_used = r.tier_used;
  if (latency_s) *latency_s = r.t_done - r.t_submit;
  sv->results.erase(it);
  return 0;
}

// Wait (bounded) until nothing is pending or in flight.  Returns 0, or
// cudaErrorTimeout when `timeout_s` elapsed first.
int gbs_server_drain(gbs_server* sv, double timeout_s) {
  if (!sv) return fail(cudaErrorInvalidValue, "null server");
  const double t0 = now_s();
  for (;;) {
    {
      std::lock_guard<std::mutex> lk(sv->mu);
      if (sv->pending.empty() && sv->in_flight == 0) return sv->error ? fail(sv->error, sv->error_msg) : 0;
    }
    if (now_s() - t0 > timeout_s) return fail(cudaErrorTimeout, "server drain timed out");
    std::this_thread::sleep_for(std::chrono::microseconds(200));
  }
}

int gbs_server_stats(gbs_server* sv, long long* completed, long long* batches, long long* pending) {
  if (!sv) return fail(cudaErrorInvalidValue, "null server");
  std::lock_guard<std::mutex> lk(sv->mu);
  if (completed) *completed = sv->completed;
  if (batches) *batches = sv->batches;
  if (pending) *pending = (long long)sv->pending.size() + sv->in_flight;
  return 0;
}

}  // extern "C"
