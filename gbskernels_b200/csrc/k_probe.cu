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
