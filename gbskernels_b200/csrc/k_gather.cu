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

// Device-resident results: scatter of a plan's results from instance order (the
// session's result arrays, grouped per launch) to request order in a caller-owned
// device block, with no host round trip.  map[k] = destination index of instance k;
// trivial requests (n = 0, odd hafnian) come as (index, re, im, aux).  A non-ok
// status carries a NaN value (the work-item kernel already wrote it; the host
// path applies the same convention).  Reference counterpart of the resident
// output: core/host_api.cu:600-658 (gbs_session_evaluate_resident).
struct ScatterArgs {
  const double* out;
  const double* aux;
  const int* st;
  const int* map;
  int ni;
  const int* tidx;
  const double* tval;  // 3 per trivial request: re, im, aux
  int ntriv;
  double* dval;        // complex, request order
  double* daux;
  int* dst;
  int write_aux;
};

__global__ void __launch_bounds__(256) scatter_kernel(ScatterArgs a) {
  const int total = a.ni + a.ntriv;
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < total; k += gridDim.x * blockDim.x) {
    int i, st;
    double re, im, x;
    if (k < a.ni) {
      i = a.map[k];
      st = a.st[k];
      re = a.out[2 * (size_t)k];
      im = a.out[2 * (size_t)k + 1];
      x = a.aux[k];
      if (st != 0) re = im = __longlong_as_double(0x7ff8000000000000ll);
    } else {
      const int t = k - a.ni;
      i = a.tidx[t];
      st = 0;
      re = a.tval[3 * t];
      im = a.tval[3 * t + 1];
      x = a.tval[3 * t + 2];
    }
    a.dval[2 * (size_t)i] = re;
    a.dval[2 * (size_t)i + 1] = im;
    if (a.write_aux) a.daux[i] = x;
    a.dst[i] = st;
  }
}

cudaError_t launch_scatter(const ScatterArgs& a, cudaStream_t st) {
  const int total = a.ni + a.ntriv;
  if (total <= 0) return cudaSuccess;
  const int grid = (total + 255) / 256 < 1184 ? (total + 255) / 256 : 1184;
  scatter_kernel<<<grid, 256, 0, st>>>(a);
  return cudaGetLastError();
}

}  // namespace gbsb
