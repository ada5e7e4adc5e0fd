// FP64 diagnostics of a state: elastic energy, per-field sum of squares and max
// |value|.  The reference has no diagnostics; these define the energy-norm drift
// and the norms reported beside each result.  Every node's contribution is
// formed and summed in double regardless of the storage precision.
#include "le2d_kernels.h"

namespace le2d {

namespace {

constexpr int kThreads = 256;

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
__device__ __forceinline__ double warp_max(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}

// out[0] += sum of energy densities, out[1+k] += sum v_k^2, out[6+k] = max |v_k| (the
// bits of a non-negative double order like the double, so an integer max works).
template <typename T>
__global__ void __launch_bounds__(kThreads) diag_kernel(const T* __restrict__ soa, int nx, int ny,
                                                        long long pitch, long long plane,
                                                        double rho, double a_nn, double a_xy,
                                                        double a_s, double* __restrict__ out) {
  double acc[11];
#pragma unroll
  for (int k = 0; k < 11; ++k) acc[k] = 0.0;
  const long long n = (long long)nx * ny;
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n;
       q += (long long)gridDim.x * blockDim.x) {
    const long long j = q / nx, i = q - j * nx;
    const T* s = soa + j * pitch + i;
    double v[NF];
#pragma unroll
    for (int k = 0; k < NF; ++k) {
      v[k] = (double)s[k * plane];
      acc[1 + k] += v[k] * v[k];
      acc[6 + k] = fmax(acc[6 + k], fabs(v[k]));
    }
    acc[0] += 0.5 * rho * (v[VX] * v[VX] + v[VY] * v[VY]) +
              a_nn * (v[SXX] * v[SXX] + v[SYY] * v[SYY]) + a_xy * v[SXX] * v[SYY] +
              a_s * v[SXY] * v[SXY];
  }
  __shared__ double red[kThreads / 32][11];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
  for (int k = 0; k < 11; ++k) {
    const double r = k < 6 ? warp_sum(acc[k]) : warp_max(acc[k]);
    if (lane == 0) red[wid][k] = r;
  }
  __syncthreads();
  if (threadIdx.x < 11) {
    const int k = threadIdx.x;
    double r = red[0][k];
    for (int w = 1; w < kThreads / 32; ++w) r = k < 6 ? r + red[w][k] : fmax(r, red[w][k]);
    if (k < 6)
      atomicAdd(out + k, r);
    else
      atomicMax(reinterpret_cast<unsigned long long*>(out + k), (unsigned long long)__double_as_longlong(r));
  }
}

}  // namespace

template <typename T>
cudaError_t launch_diag(const T* soa, int nx, int ny, long long pitch, long long plane,
                        double rho, double a_nn, double a_xy, double a_s, double* out,
                        cudaStream_t s) {
  long long blocks = ((long long)nx * ny + kThreads - 1) / kThreads;
  if (blocks > 148LL * 8) blocks = 148LL * 8;
  if (blocks < 1) blocks = 1;
  diag_kernel<T><<<(int)blocks, kThreads, 0, s>>>(soa, nx, ny, pitch, plane, rho, a_nn, a_xy, a_s,
                                                  out);
  return cudaGetLastError();
}

template cudaError_t launch_diag<float>(const float*, int, int, long long, long long, double,
                                        double, double, double, double*, cudaStream_t);
template cudaError_t launch_diag<double>(const double*, int, int, long long, long long, double,
                                         double, double, double, double*, cudaStream_t);

}  // namespace le2d
