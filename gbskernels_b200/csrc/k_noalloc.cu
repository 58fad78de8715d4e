// k_noalloc.cu -- a hafnian entry point that allocates nothing.
//
// Some callers cannot call cudaMalloc at evaluation time: a process whose device
// memory is owned by another allocator (a framework's caching pool that must see
// every allocation), a latency-critical loop where an allocation would synchronise
// the device, or an embedded host that forbids dynamic allocation after start-up.
// gbs_haf_noalloc serves them: the
// caller passes device pointers to the input matrices and the output vector, and
// every scratch buffer the hafnian work-item kernel needs (work queue, per-item
// partials, completion counters, per-instance side outputs) lives in one
// file-scope __device__ array of fixed size, kNoAllocScratchBytes (4 MiB), that
// every GPU loading this library holds until the process exits.
//
// The work queue is written on the device by a small fill kernel (each descriptor
// is a pure function of the instance index, N and the split), which also clears
// the queue head and the completion counters: no host staging buffer and no
// host-to-device copy is involved, so nothing the call leaves behind on the host
// can be read by the GPU later.
//
// The result equals gbs_haf_host's bit for bit for complex input (same work items,
// same kernel).  Every input here takes the complex power loop; gbs_haf_host runs
// a real input (every imaginary part zero) through the real loop, so for real
// input the two agree to rounding.
#include <cuda_runtime.h>

#include <cstdio>
#include <mutex>

#include "gbs_items.cuh"

namespace gbsb {

int tuned_split(int fn, int tier, int dim);  // host_api.cu: the autotuner's split table

// Fixed scratch: 4 MiB per device, 256-byte aligned.
constexpr size_t kNoAllocScratchBytes = (size_t)4 << 20;
// Limits that fit the scratch: items x 68 bytes + instances x 48 bytes + 256.
constexpr int kNoAllocMaxInstances = 16384;
constexpr int kNoAllocMaxItems = 49152;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

// One thread per work item writes its WorkItem; the first item of an instance also
// writes the InstDesc and clears the instance's completion counter; thread 0 clears
// the queue head.  Grid-stride, so any grid covers every item.
__global__ void noalloc_fill_queue(InstDesc* insts, WorkItem* items, int* done, int* head, int batch, int N,
                                   int per, int items_per) {
  const long long nit = (long long)batch * items_per;
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x; k < nit; k += stride) {
    const int b = (int)(k / items_per);
    const int j = (int)(k - (long long)b * items_per);
    WorkItem w{};
    w.inst = b;
    w.lo = (unsigned long long)j << per;
    w.count = 1ull << per;
    items[k] = w;
    if (j == 0) {
      InstDesc d{};
      d.off = (long long)b * 2 * N * N;
      d.dim = N;
      d.ft = ft_code(kFnHaf, kTierFp64);
      d.item0 = (int)k;
      d.nitems = items_per;
      insts[b] = d;
      done[b] = 0;
    }
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) *head = 0;
}

// haf of the empty matrix is 1, of an odd-sided one 0: written straight to d_out.
__global__ void noalloc_fill_trivial(double* out, int batch, double value) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < batch; i += gridDim.x * blockDim.x) {
    out[2 * i] = value;
    out[2 * i + 1] = 0.0;
  }
}

namespace {

constexpr int kMaxDevices = 64;
std::mutex g_noalloc_mu;
void* g_scratch_ptr[kMaxDevices] = {};  // device address of g_noalloc_scratch, per device
char g_noalloc_err[256] = "";  // static: the error path allocates nothing either
void set_err(const char* m) { std::snprintf(g_noalloc_err, sizeof(g_noalloc_err), "%s", m); }

size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }

// Device address of the scratch array for the current device, looked up once per
// device with that device current (the symbol's host name is only a stand-in).
cudaError_t scratch_for_current_device(void** out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev < 0 || dev >= kMaxDevices) return cudaErrorInvalidDevice;
  if (!g_scratch_ptr[dev]) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) return e;
    g_scratch_ptr[dev] = p;
  }
  *out = g_scratch_ptr[dev];
  return cudaSuccess;
}

}  // namespace
}  // namespace gbsb

using namespace gbsb;

extern "C" {

// Hafnians of `batch` symmetric N x N complex matrices (interleaved binary64,
// row-major, batch-contiguous) already on the device at d_mats, written to d_out
// (batch complex values), on `stream` (a cudaStream_t; NULL = legacy default).
// Allocates nothing: the scratch is the fixed 4 MiB array above.
//  * Limits: N <= 32, batch <= 16384 and at most 49152 work items.  The item count
//    is batch x 2^(N/2 - split) for the split in force for (haf, fp64, N): 7 by
//    default (so batch x 2^max(0, N/2 - 7)), or the autotuner's value after
//    gbs_set_split -- the same split gbs_haf_host uses, which keeps the values
//    equal.  Larger requests return cudaErrorInvalidValue before any launch.
//  * The first call on a device looks up the scratch array's device address
//    (cudaGetSymbolAddress, with that device current) and keeps it.
//  * Every call shares the one array and keeps the last call's contents (the fill
//    kernel rewrites the queue and clears the counters each call); calls whose
//    executions overlap on the GPU (different streams, or threads racing on one
//    stream) corrupt each other -- serialise them.
//  * Asynchronous on `stream`: two kernel launches, no copies.
int gbs_haf_noalloc(const double* d_mats, int N, int batch, double* d_out, void* stream) {
  std::lock_guard<std::mutex> lk(g_noalloc_mu);
  cudaStream_t st = (cudaStream_t)stream;
  if (batch < 0 || N < 0) { set_err("gbs_haf_noalloc: negative size"); return (int)cudaErrorInvalidValue; }
  if (batch == 0) return 0;
  // an empty matrix (N = 0) has no entries to read: its input pointer may be null
  if (!d_out || (!d_mats && N > 0)) { set_err("gbs_haf_noalloc: null device pointer"); return (int)cudaErrorInvalidValue; }
  if (N > kHafMaxN) { set_err("gbs_haf_noalloc: N above 32"); return (int)cudaErrorInvalidValue; }
  if (batch > kNoAllocMaxInstances) {
    set_err("gbs_haf_noalloc: batch above 16384");
    return (int)cudaErrorInvalidValue;
  }
  if (N == 0 || (N & 1)) {
    noalloc_fill_trivial<<<(batch + 255) / 256, 256, 0, st>>>(d_out, batch, N == 0 ? 1.0 : 0.0);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) set_err("gbs_haf_noalloc: launch failed");
    return (int)e;
  }
  const int n = N / 2;
  int per = n < kHafItemLog2 ? n : kHafItemLog2;  // the planner's decomposition (bit-identical results)
  const int tl = tuned_split(kFnHaf, kTierFp64, N);
  if (tl >= 0) per = tl < n ? tl : n;
  const long long items_per = 1ll << (n - per);
  const long long nit = items_per * batch;
  if (nit > kNoAllocMaxItems) {
    std::snprintf(g_noalloc_err, sizeof(g_noalloc_err),
                  "gbs_haf_noalloc: %d instances x %lld items = %lld work items exceed the fixed "
                  "scratch (max 49152 items)", batch, items_per, nit);
    return (int)cudaErrorInvalidValue;
  }
  void* base = nullptr;
  cudaError_t e = scratch_for_current_device(&base);
  if (e != cudaSuccess) { set_err("gbs_haf_noalloc: cudaGetSymbolAddress failed"); return (int)e; }
  // carve the scratch
  char* p = (char*)base;
  size_t o = 0;
  InstDesc* d_insts = (InstDesc*)(p + o); o = align256(o + sizeof(InstDesc) * batch);
  WorkItem* d_items = (WorkItem*)(p + o); o = align256(o + sizeof(WorkItem) * nit);
  double* d_part = (double*)(p + o); o = align256(o + sizeof(double) * 4 * nit);
  double* d_paux = (double*)(p + o); o = align256(o + sizeof(double) * nit);
  int* d_pst = (int*)(p + o); o = align256(o + sizeof(int) * nit);
  int* d_done = (int*)(p + o); o = align256(o + sizeof(int) * batch);
  int* d_head = (int*)(p + o); o = align256(o + 64);
  double* d_aux = (double*)(p + o); o = align256(o + sizeof(double) * batch);
  int* d_st = (int*)(p + o); o = align256(o + sizeof(int) * batch);
  if (o > kNoAllocScratchBytes) { set_err("gbs_haf_noalloc: scratch layout overflow"); return (int)cudaErrorInvalidValue; }
  // the work queue, the completion counters and the queue head, written on the device
  const int fill_grid = (int)std::min<long long>((nit + 255) / 256, 1024);
  noalloc_fill_queue<<<fill_grid, 256, 0, st>>>(d_insts, d_items, d_done, d_head, batch, N, per, (int)items_per);
  e = cudaGetLastError();
  if (e != cudaSuccess) { set_err("gbs_haf_noalloc: queue fill launch failed"); return (int)e; }
  ItemLaunch L{};
  L.mats = d_mats;
  L.insts = d_insts;
  L.items = d_items;
  L.order = nullptr;
  L.n_items = (int)nit;
  L.head = d_head;
  L.done = d_done;
  L.part = d_part;
  L.paux = d_paux;
  L.pst = d_pst;
  L.out = d_out;
  L.aux_out = d_aux;
  L.st_out = d_st;
  L.haf_smax = N;
  L.ws_doubles = (haf_layout(N).total + 3) & ~3;
  constexpr unsigned BR = br1(kFnHaf, kTierFp64);
  const int bps = occ_br<BR>(L, 1);
  int dev = 0, sms = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  if (bps <= 0) { set_err("gbs_haf_noalloc: kernel does not fit on an SM"); return (int)cudaErrorInvalidConfiguration; }
  const int grid = (int)std::min<long long>((long long)sms * bps, nit);
  e = launch_br<BR>(L, grid, 1, st);
  if (e != cudaSuccess) { set_err("gbs_haf_noalloc: kernel launch failed"); return (int)e; }
  return 0;
}

const char* gbs_haf_noalloc_last_error(void) { return g_noalloc_err; }

}  // extern "C"
