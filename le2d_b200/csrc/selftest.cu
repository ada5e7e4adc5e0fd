// Self-test of the FP64 slope-ratio division used by the step kernels (ratio(double) in
// le2d_device.cuh) against CUDA's IEEE division, operand pair by operand pair on the
// device.  Test surface only: the step does not call it.
#include <cstdio>

#include "le2d.h"
#include "le2d_kernels.h"

namespace le2d {
namespace {

__global__ void ratio_kernel(const double* __restrict__ a, const double* __restrict__ b, long long n,
                             double* __restrict__ fast, double* __restrict__ ieee) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    fast[i] = ratio(a[i], b[i]);
    ieee[i] = __ddiv_rn(a[i], b[i]);
  }
}

}  // namespace
}  // namespace le2d

extern "C" int le2d_selftest_ratio(const double* a, const double* b, long long n, double* fast,
                                   double* ieee) {
  if (n < 0 || (n > 0 && (!a || !b || !fast || !ieee))) return LE2D_EINVAL;
  if (n == 0) return LE2D_OK;
  const size_t bytes = (size_t)n * sizeof(double);
  double* d = nullptr;
  if (cudaMalloc(&d, 4 * bytes) != cudaSuccess) {
    cudaGetLastError();
    return LE2D_ENOMEM;
  }
  double *da = d, *db = d + n, *df = d + 2 * n, *di = d + 3 * n;
  cudaError_t e = cudaMemcpy(da, a, bytes, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(db, b, bytes, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) {
    long long blocks = (n + 255) / 256;
    if (blocks > 4096) blocks = 4096;
    le2d::ratio_kernel<<<(int)blocks, 256>>>(da, db, n, df, di);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaMemcpy(fast, df, bytes, cudaMemcpyDeviceToHost);
  if (e == cudaSuccess) e = cudaMemcpy(ieee, di, bytes, cudaMemcpyDeviceToHost);
  cudaFree(d);
  if (e != cudaSuccess) {
    fprintf(stderr, "le2d_selftest_ratio: %s\n", cudaGetErrorString(e));
    return LE2D_ECUDA;
  }
  return LE2D_OK;
}
