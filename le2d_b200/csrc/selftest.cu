// Self-tests of the FP64 slope-ratio division used by the step kernels (ratio(double) in
// le2d_device.cuh) against CUDA's IEEE division, and of the limited slope ratio the FP64
// step computes (psi_ratio: the division fused with the superbee limiter), operand pair by
// operand pair on the device.  Test surface only: the step does not call them.
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

__global__ void limiter_kernel(const double* __restrict__ a, const double* __restrict__ b, double kc,
                               long long n, double* __restrict__ out) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x)
    out[i] = psi_ratio(a[i], b[i], kc);
}

// Copies n doubles of each host input to the device, runs `launch` on the device copies,
// copies `nout` output arrays back.
template <typename F>
int run_selftest(const char* name, const double* const* in, int nin, double* const* out, int nout,
                 long long n, F launch) {
  const size_t bytes = (size_t)n * sizeof(double);
  double* d = nullptr;
  if (cudaMalloc(&d, (size_t)(nin + nout) * bytes) != cudaSuccess) {
    cudaGetLastError();
    return LE2D_ENOMEM;
  }
  cudaError_t e = cudaSuccess;
  for (int k = 0; k < nin && e == cudaSuccess; ++k) e = cudaMemcpy(d + k * n, in[k], bytes, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) {
    long long blocks = (n + 255) / 256;
    if (blocks > 4096) blocks = 4096;
    launch((int)blocks, d, d + nin * n);
    e = cudaGetLastError();
  }
  for (int k = 0; k < nout && e == cudaSuccess; ++k)
    e = cudaMemcpy(out[k], d + (nin + k) * n, bytes, cudaMemcpyDeviceToHost);
  cudaFree(d);
  if (e != cudaSuccess) {
    fprintf(stderr, "%s: %s\n", name, cudaGetErrorString(e));
    return LE2D_ECUDA;
  }
  return LE2D_OK;
}

}  // namespace
}  // namespace le2d

extern "C" int le2d_selftest_ratio(const double* a, const double* b, long long n, double* fast,
                                   double* ieee) {
  if (n < 0 || (n > 0 && (!a || !b || !fast || !ieee))) return LE2D_EINVAL;
  if (n == 0) return LE2D_OK;
  const double* in[2] = {a, b};
  double* out[2] = {fast, ieee};
  return le2d::run_selftest("le2d_selftest_ratio", in, 2, out, 2, n, [&](int blocks, double* d, double* o) {
    le2d::ratio_kernel<<<blocks, 256>>>(d, d + n, n, o, o + n);
  });
}

extern "C" int le2d_selftest_limiter(const double* a, const double* b, double kc, long long n, double* out) {
  if (n < 0 || (n > 0 && (!a || !b || !out))) return LE2D_EINVAL;
  if (n == 0) return LE2D_OK;
  const double* in[2] = {a, b};
  double* outs[1] = {out};
  return le2d::run_selftest("le2d_selftest_limiter", in, 2, outs, 1, n, [&](int blocks, double* d, double* o) {
    le2d::limiter_kernel<<<blocks, 256>>>(d, d + n, kc, n, o);
  });
}
