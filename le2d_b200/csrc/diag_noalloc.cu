// Diagnostics of a caller-held device state without any allocation.
//
// Some callers cannot allocate device memory: hosts that budget all device memory up
// front (e.g. a serving loop with a fixed arena, where any extra cudaMalloc would escape
// the budget), or time loops where a cudaMalloc/cudaFree would synchronise the device.
// This entry point needs no task and allocates nothing: its scratch is the file-scope
// device array below, sized for at most LE2D_DIAG_NOALLOC_MAX_ROWS grid rows.
//
// The array is held by every GPU that loads the library until the process exits.  All
// calls share it and it keeps the last call's contents; pass 1 overwrites every partial
// it uses and pass 2 overwrites the result, so nothing has to start at zero.  Calls whose
// kernels overlap on the GPU race on it (issue them in one stream or synchronise).
#include <cstdio>
#include <mutex>

#include "le2d.h"
#include "le2d_kernels.h"

namespace {

constexpr int kNoallocRows = LE2D_DIAG_NOALLOC_MAX_ROWS;
constexpr int kVals = 11;  // energy, 5 sums of squares, 5 max |value|
constexpr int kThreads = 256;

// [row][11] partials of pass 1, then the 11 results of pass 2.
static __device__ __align__(256) double g_diag_scratch[(kNoallocRows + 1) * kVals];

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

// Reduces acc[11] over the block (sums for 0..5, max for 6..10) into out[0..10].
__device__ __forceinline__ void block_reduce(double (&acc)[kVals], double* out) {
  __shared__ double red[kThreads / 32][kVals];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
  for (int k = 0; k < kVals; ++k) {
    const double r = k < 6 ? warp_sum(acc[k]) : warp_max(acc[k]);
    if (lane == 0) red[wid][k] = r;
  }
  __syncthreads();
  if (threadIdx.x < kVals) {
    const int k = threadIdx.x;
    double r = red[0][k];
    for (int w = 1; w < kThreads / 32; ++w) r = k < 6 ? r + red[w][k] : fmax(r, red[w][k]);
    out[k] = r;
  }
}

// Pass 1: block j reduces row j into scratch[j][*].
__global__ void __launch_bounds__(kThreads)
    diag_rows_kernel(const real* __restrict__ soa, int nx, long long pitch, long long plane,
                     double rho, double a_nn, double a_xy, double a_s, double* scratch) {
  double acc[kVals];
#pragma unroll
  for (int k = 0; k < kVals; ++k) acc[k] = 0.0;
  const real* row = soa + (long long)blockIdx.x * pitch;
  for (int i = threadIdx.x; i < nx; i += kThreads) {
    double v[5];
#pragma unroll
    for (int k = 0; k < 5; ++k) {
      v[k] = (double)row[k * plane + i];
      acc[1 + k] += v[k] * v[k];
      acc[6 + k] = fmax(acc[6 + k], fabs(v[k]));
    }
    acc[0] += 0.5 * rho * (v[0] * v[0] + v[1] * v[1]) + a_nn * (v[2] * v[2] + v[4] * v[4]) +
              a_xy * v[2] * v[4] + a_s * v[3] * v[3];
  }
  block_reduce(acc, scratch + (long long)blockIdx.x * kVals);
}

// Pass 2: one block reduces the ny row partials in a fixed order into scratch[kNoallocRows][*].
__global__ void __launch_bounds__(kThreads) diag_final_kernel(int ny, double* scratch) {
  double acc[kVals];
#pragma unroll
  for (int k = 0; k < kVals; ++k) acc[k] = 0.0;
  for (int j = threadIdx.x; j < ny; j += kThreads) {
#pragma unroll
    for (int k = 0; k < kVals; ++k) {
      const double x = scratch[(long long)j * kVals + k];
      acc[k] = k < 6 ? acc[k] + x : fmax(acc[k], x);
    }
  }
  block_reduce(acc, scratch + (long long)kNoallocRows * kVals);
}

// Device address of g_diag_scratch per device, looked up with that device current (a
// host-side use of the symbol's name is only a stand-in, not a device address): once per
// device and context -- a reset of the device (cudaDeviceReset) destroys the context whose
// address was cached, and the next call looks it up again in the new one.
std::mutex g_mu;
double* g_addr[64] = {nullptr};
unsigned long long g_ctx[64] = {0};

// The current context's unique id (driver API cuCtxGetCurrent / cuCtxGetId, reached through
// the runtime's entry-point query so the library needs no link to the driver library), or 0
// when unavailable -- then the address is looked up on every call.
unsigned long long context_id() {
  using GetCurrent = int (*)(void**);
  using GetId = int (*)(void*, unsigned long long*);
  static GetCurrent get_current = nullptr;
  static GetId get_id = nullptr;
  static bool tried = false;
  if (!tried) {  // under g_mu
    tried = true;
    void* f1 = nullptr;
    void* f2 = nullptr;
    cudaDriverEntryPointQueryResult q1, q2;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f1, cudaEnableDefault, &q1) == cudaSuccess &&
        cudaGetDriverEntryPoint("cuCtxGetId", &f2, cudaEnableDefault, &q2) == cudaSuccess &&
        q1 == cudaDriverEntryPointSuccess && q2 == cudaDriverEntryPointSuccess) {
      get_current = reinterpret_cast<GetCurrent>(f1);
      get_id = reinterpret_cast<GetId>(f2);
    }
    cudaGetLastError();
  }
  void* ctx = nullptr;
  unsigned long long id = 0;
  if (!get_current || !get_id || get_current(&ctx) != 0 || !ctx || get_id(ctx, &id) != 0) return 0;
  return id;
}

}  // namespace

extern "C" int le2d_diagnostics_noalloc(const real* d_state, int nx, int ny, long long pitch,
                                        long long plane, real hx, real hy, real c1, real c2,
                                        real rho, void* stream, le2d_diag_t* out) {
  if (!d_state || !out || nx < 1 || ny < 1 || pitch < nx || plane < pitch * ny) {
    fprintf(stderr, "le2d: le2d_diagnostics_noalloc: bad arguments\n");
    return LE2D_EINVAL;
  }
  if (ny > kNoallocRows) {
    fprintf(stderr,
            "le2d: le2d_diagnostics_noalloc: %d rows exceed the static scratch of %d rows "
            "(use le2d_diagnostics)\n",
            ny, kNoallocRows);
    return LE2D_EINVAL;
  }
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess || dev < 0 || dev >= 64) {
    fprintf(stderr, "le2d: le2d_diagnostics_noalloc: no CUDA device\n");
    return LE2D_ENODEV;
  }
  double* scratch = nullptr;
  {
    std::lock_guard<std::mutex> lk(g_mu);
    const unsigned long long ctx = context_id();  // 0 before the device's context exists
    if (!g_addr[dev] || ctx == 0 || ctx != g_ctx[dev]) {
      g_ctx[dev] = ctx;
      e = cudaGetSymbolAddress((void**)&g_addr[dev], g_diag_scratch);
      if (e != cudaSuccess) {
        g_addr[dev] = nullptr;
        fprintf(stderr, "le2d: le2d_diagnostics_noalloc: cudaGetSymbolAddress: %s\n",
                cudaGetErrorString(e));
        return LE2D_ECUDA;
      }
    }
    scratch = g_addr[dev];
  }
  const cudaStream_t s = (cudaStream_t)stream;
  const double r = rho, a = c1, b = c2;
  const double mu = r * b * b, la = r * a * a - 2.0 * mu;
  diag_rows_kernel<<<ny, kThreads, 0, s>>>(d_state, nx, pitch, plane, r,
                                           (la + 2.0 * mu) / (8.0 * mu * (la + mu)),
                                           -2.0 * la / (8.0 * mu * (la + mu)), 1.0 / (2.0 * mu),
                                           scratch);
  diag_final_kernel<<<1, kThreads, 0, s>>>(ny, scratch);
  double h[kVals];
  e = cudaGetLastError();
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(h, scratch + (long long)kNoallocRows * kVals, sizeof(h),
                        cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) {
    fprintf(stderr, "le2d: le2d_diagnostics_noalloc: %s\n", cudaGetErrorString(e));
    return LE2D_ECUDA;
  }
  out->energy = h[0] * (double)hx * (double)hy;
  for (int k = 0; k < 5; ++k) {
    out->sumsq[k] = h[1 + k];
    out->maxabs[k] = h[6 + k];
  }
  return LE2D_OK;
}
