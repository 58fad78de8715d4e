// k_probe.cu -- FP64 tensor-core throughput probe (the roofline denominator).
//
// Independent mma.sync m16n8k8 (or m16n8k4) .f64 chains (8 accumulators per warp,
// no memory traffic), one launch filling every SM: the sustained FP64 rate the
// work-item kernels are measured against.  Used by bench.py; never on the
// evaluation path.
#include <cuda_runtime.h>

#include <cstdint>

namespace gbsb {

template <int K>
__global__ void __launch_bounds__(128) fp64_mma_probe_kernel(double* sink, int iters) {
  double a[4], b[2], c[8][4];
#pragma unroll
  for (int i = 0; i < 4; ++i) a[i] = 1.0 + 1e-3 * (threadIdx.x + i);
#pragma unroll
  for (int i = 0; i < 2; ++i) b[i] = 1.0 - 1e-3 * (threadIdx.x + i);
#pragma unroll
  for (int t = 0; t < 8; ++t) c[t][0] = c[t][1] = c[t][2] = c[t][3] = 0.0;
  for (int it = 0; it < iters; ++it) {
#pragma unroll
    for (int t = 0; t < 8; ++t) {
      if constexpr (K == 8) {
        asm volatile(
            "mma.sync.aligned.m16n8k8.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
            "{%0,%1,%2,%3};\n"
            : "+d"(c[t][0]), "+d"(c[t][1]), "+d"(c[t][2]), "+d"(c[t][3])
            : "d"(a[0]), "d"(a[1]), "d"(a[2]), "d"(a[3]), "d"(b[0]), "d"(b[1]));
      } else {
        asm volatile(
            "mma.sync.aligned.m16n8k4.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, {%4,%5}, {%6}, {%0,%1,%2,%3};\n"
            : "+d"(c[t][0]), "+d"(c[t][1]), "+d"(c[t][2]), "+d"(c[t][3])
            : "d"(a[0]), "d"(a[1]), "d"(b[0]));
      }
    }
  }
  double s = 0.0;
#pragma unroll
  for (int t = 0; t < 8; ++t) s += c[t][0] + c[t][1] + c[t][2] + c[t][3];
  if (s == 1234.5678) sink[0] = s;  // never true; keeps the chains live
}

}  // namespace gbsb

template <int K>
static int probe(double* tflops, float* ms_out) {
  int dev = 0, sms = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  double* sink = nullptr;
  if (e == cudaSuccess) e = cudaMalloc(&sink, sizeof(double));
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  if (e == cudaSuccess) e = cudaEventCreate(&e0);
  if (e == cudaSuccess) e = cudaEventCreate(&e1);
  const int blocks = sms * 2, iters = 4000;
  float ms = 0.f;
  if (e == cudaSuccess) {
    gbsb::fp64_mma_probe_kernel<K><<<blocks, 128>>>(sink, 50);
    cudaEventRecord(e0);
    gbsb::fp64_mma_probe_kernel<K><<<blocks, 128>>>(sink, iters);
    cudaEventRecord(e1);
    e = cudaEventSynchronize(e1);
  }
  if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, e0, e1);
  if (e == cudaSuccess) {
    const double flops = 2.0 * 16 * 8 * K * 8.0 * iters * (double)blocks * 4.0;  // 8 mma x 4 warps per block
    if (tflops) *tflops = flops / (ms * 1e-3) / 1e12;
    if (ms_out) *ms_out = ms;
  }
  if (e0) cudaEventDestroy(e0);
  if (e1) cudaEventDestroy(e1);
  if (sink) cudaFree(sink);
  return (int)e;
}

extern "C" int gbs_probe_fp64_peak(double* tflops, float* ms_out) { return probe<8>(tflops, ms_out); }
extern "C" int gbs_probe_fp64_mma(int k, double* tflops, float* ms_out) {
  if (k == 4) return probe<4>(tflops, ms_out);
  if (k == 8) return probe<8>(tflops, ms_out);
  return (int)cudaErrorInvalidValue;
}

namespace gbsb {

// T independent m16n8k8 (K = 8) or m16n8k4 (K = 4) chains per warp, `iters` steps;
// warp 0 of block 0 records the cycles the loop took (clock64), so that cycles /
// (iters T) is the issue interval of one mma and, for T = 1, its latency.
template <int T, int K>
__global__ void fp64_mma_chains_kernel(double* sink, long long* cyc, int iters) {
  double a[4], b[2], c[T][4];
#pragma unroll
  for (int i = 0; i < 4; ++i) a[i] = 1.0 + 1e-9 * (threadIdx.x + i);
#pragma unroll
  for (int i = 0; i < 2; ++i) b[i] = 1.0 - 1e-9 * (threadIdx.x + i);
#pragma unroll
  for (int t = 0; t < T; ++t) c[t][0] = c[t][1] = c[t][2] = c[t][3] = 0.0;
  __syncthreads();
  const long long t0 = clock64();
  for (int it = 0; it < iters; ++it) {
#pragma unroll
    for (int t = 0; t < T; ++t) {
      if constexpr (K == 8) {
        asm volatile(
            "mma.sync.aligned.m16n8k8.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
            "{%0,%1,%2,%3};\n"
            : "+d"(c[t][0]), "+d"(c[t][1]), "+d"(c[t][2]), "+d"(c[t][3])
            : "d"(a[0]), "d"(a[1]), "d"(a[2]), "d"(a[3]), "d"(b[0]), "d"(b[1]));
      } else {
        asm volatile(
            "mma.sync.aligned.m16n8k4.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, {%4,%5}, {%6}, {%0,%1,%2,%3};\n"
            : "+d"(c[t][0]), "+d"(c[t][1]), "+d"(c[t][2]), "+d"(c[t][3])
            : "d"(a[0]), "d"(a[1]), "d"(b[0]));
      }
    }
  }
  double s = 0.0;
#pragma unroll
  for (int t = 0; t < T; ++t) s += c[t][0] + c[t][1] + c[t][2] + c[t][3];
  const long long t1 = clock64();  // after the sum: the chains have completed
  if (s == 1234.5678) sink[0] = s;
  if (threadIdx.x == 0 && blockIdx.x == 0) cyc[0] = t1 - t0;
}

}  // namespace gbsb

template <int T, int K>
static int chains(int warps_per_block, int blocks, double* tflops, double* cycles) {
  double* sink = nullptr;
  long long* cyc = nullptr;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  cudaError_t e = cudaMalloc(&sink, 64);
  if (e == cudaSuccess) e = cudaMalloc(&cyc, 64);
  if (e == cudaSuccess) e = cudaEventCreate(&e0);
  if (e == cudaSuccess) e = cudaEventCreate(&e1);
  const int iters = 2000;
  float ms = 0.f;
  if (e == cudaSuccess) {
    gbsb::fp64_mma_chains_kernel<T, K><<<blocks, 32 * warps_per_block>>>(sink, cyc, 10);
    cudaEventRecord(e0);
    gbsb::fp64_mma_chains_kernel<T, K><<<blocks, 32 * warps_per_block>>>(sink, cyc, iters);
    cudaEventRecord(e1);
    e = cudaEventSynchronize(e1);
  }
  if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, e0, e1);
  long long c = 0;
  if (e == cudaSuccess) e = cudaMemcpy(&c, cyc, sizeof(c), cudaMemcpyDeviceToHost);
  if (e == cudaSuccess) {
    const double flops = 2.0 * 16 * 8 * K * (double)T * iters * warps_per_block * (double)blocks;
    if (tflops) *tflops = flops / (ms * 1e-3) / 1e12;
    if (cycles) *cycles = (double)c / ((double)iters * T);
  }
  if (e0) cudaEventDestroy(e0);
  if (e1) cudaEventDestroy(e1);
  if (sink) cudaFree(sink);
  if (cyc) cudaFree(cyc);
  return (int)e;
}

// Shape sweep of the probe: k = 8 or 4, `chains` in {1, 2, 4, 8} independent
// accumulator chains per warp, warps_per_block warps (1..16) in each of `blocks`
// blocks (one per SM for a per-SM figure); *cycles = warp 0's cycles per mma.
extern "C" int gbs_probe_fp64_mma_chains(int k, int chains_per_warp, int warps_per_block, int blocks, double* tflops,
                                        double* cycles) {
  if (warps_per_block < 1 || warps_per_block > 16 || blocks < 1) return (int)cudaErrorInvalidValue;
#define GBSB_CH(T)                                                                     \
  if (chains_per_warp == T) {                                                          \
    if (k == 8) return chains<T, 8>(warps_per_block, blocks, tflops, cycles);          \
    if (k == 4) return chains<T, 4>(warps_per_block, blocks, tflops, cycles);          \
  }
  GBSB_CH(1) GBSB_CH(2) GBSB_CH(4) GBSB_CH(8)
#undef GBSB_CH
  return (int)cudaErrorInvalidValue;
}
