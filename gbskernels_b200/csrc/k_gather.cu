// k_gather.cu -- on-device gather of resident-state submatrices for the serving
// loop: out = state[idx][:, idx] (M x M complex state resident in HBM), with the
// loop weights gamma[idx] on the diagonal for loop hafnians and the A (+) [1]
// augmentation for odd loop-hafnian sizes.  Reference counterpart:
// core/sampler_gather.cu:20-57 (the sampler's A_k[idx, idx] gather).
#include <cuda_runtime.h>

namespace gbsb {

struct GatherDesc {
  long long out_off;
  long long idx_off;
  const double* state;
  const double* gamma;
  int d, de, M, use_gamma;
};

__global__ void __launch_bounds__(128) gather_kernel(const GatherDesc* __restrict__ descs,
                                                     const int* __restrict__ idx, double* __restrict__ mats) {
  const GatherDesc g = descs[blockIdx.x];
  const int* ix = idx + g.idx_off;
  double2* out = reinterpret_cast<double2*>(mats + g.out_off);
  const double2* S = reinterpret_cast<const double2*>(g.state);
  const int de = g.de, d = g.d;
  for (int e = threadIdx.x; e < de * de; e += blockDim.x) {
    const int r = e / de, c = e - r * de;
    double2 v = make_double2(0.0, 0.0);
    if (r < d && c < d) {
      if (g.use_gamma && r == c) v = reinterpret_cast<const double2*>(g.gamma)[ix[r]];
      else v = S[(size_t)ix[r] * g.M + ix[c]];
    } else if (r == d && c == d) {
      v = make_double2(1.0, 0.0);  // lhaf(A) = lhaf(A (+) [1]) for odd N
    }
    out[e] = v;
  }
}

cudaError_t launch_gather(const GatherDesc* descs, int n, const int* idx, double* mats, cudaStream_t st) {
  if (n <= 0) return cudaSuccess;
  gather_kernel<<<n, 128, 0, st>>>(descs, idx, mats);
  return cudaGetLastError();
}

}  // namespace gbsb
