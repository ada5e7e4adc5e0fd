// Layout conversion between the caller's contiguous grid (the reference's AOS
// le_node array or its SoA planes, le2d simple/le_core.c:13-21) and the device's
// pitched SoA planes, and the pressure-disk initial condition on the device.
#include "le2d_kernels.h"

namespace le2d {

namespace {

template <typename T>
__global__ void pack_kernel(const T* __restrict__ raw, T* __restrict__ soa, int nx, int ny,
                            long long pitch, long long plane, int aos) {
  const long long n = (long long)nx * ny;
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n;
       q += (long long)gridDim.x * blockDim.x) {
    const long long j = q / nx, i = q - j * nx;
    T* d = soa + j * pitch + i;
#pragma unroll
    for (int k = 0; k < NF; ++k) d[k * plane] = aos ? raw[q * NF + k] : raw[k * n + q];
  }
}

template <typename T>
__global__ void unpack_kernel(const T* __restrict__ soa, T* __restrict__ raw, int nx, int ny,
                              long long pitch, long long plane, int aos) {
  const long long n = (long long)nx * ny;
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n;
       q += (long long)gridDim.x * blockDim.x) {
    const long long j = q / nx, i = q - j * nx;
    const T* s = soa + j * pitch + i;
#pragma unroll
    for (int k = 0; k < NF; ++k) {
      const T v = s[k * plane];
      if (aos)
        raw[q * NF + k] = v;
      else
        raw[k * n + q] = v;
    }
  }
}

// Products and sums rounded one at a time (no contraction), so the disk matches the
// host loop of le_set_ball bit for bit: position h*i in T, squared distance in T,
// sqrt and comparison with r in double (simple/le_core.c:76-78).
__device__ __forceinline__ float mul_rn(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ double mul_rn(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ float add_rn(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ double add_rn(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ float sub_rn(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ double sub_rn(double a, double b) { return __dsub_rn(a, b); }

template <typename T>
__global__ void set_ball_kernel(T* __restrict__ soa, int nx, int ny, long long pitch,
                                long long plane, T hx, T hy, T cx, T cy, T r, T s) {
  const long long n = (long long)nx * ny;
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n;
       q += (long long)gridDim.x * blockDim.x) {
    const int j = (int)(q / nx), i = (int)(q - (long long)j * nx);
    const T dx = sub_rn(mul_rn(hx, (T)i), cx);
    const T dy = sub_rn(mul_rn(hy, (T)j), cy);
    const T d2 = add_rn(mul_rn(dx, dx), mul_rn(dy, dy));
    if (sqrt((double)d2) < (double)r) {
      T* d = soa + (long long)j * pitch + i;
      d[SXX * plane] = s;
      d[SYY * plane] = s;
    }
  }
}

// |v| = sqrt(vx^2 + vy^2) as the reference's VTK writer stores it (simple/le_core.c:99-111,
// :150-165): the squares and their sum rounded one at a time in T, the square root in
// double (correctly rounded, as the host's sqrt), rounded to float, stored big-endian;
// nodes in the order j outer, i inner.
template <typename T>
__global__ void vtk_speed_kernel(const T* __restrict__ soa, int nx, int ny, long long pitch,
                                 long long plane, unsigned* __restrict__ out) {
  const long long n = (long long)nx * ny;
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n;
       q += (long long)gridDim.x * blockDim.x) {
    const long long j = q / nx, i = q - j * nx;
    const T* s = soa + j * pitch + i;
    const T vx = s[VX * plane], vy = s[VY * plane];
    const T s2 = add_rn(mul_rn(vx, vx), mul_rn(vy, vy));
    const float v = (float)sqrt((double)s2);
    out[q] = __byte_perm(__float_as_uint(v), 0, 0x0123);
  }
}

inline int grid_for(long long n) {
  long long b = (n + 255) / 256;
  if (b > 148LL * 16) b = 148LL * 16;
  return (int)(b < 1 ? 1 : b);
}

}  // namespace

template <typename T>
cudaError_t launch_pack(const T* raw, T* soa, int nx, int ny, long long pitch, long long plane,
                        int aos, cudaStream_t s) {
  pack_kernel<T><<<grid_for((long long)nx * ny), 256, 0, s>>>(raw, soa, nx, ny, pitch, plane, aos);
  return cudaGetLastError();
}

template <typename T>
cudaError_t launch_unpack(const T* soa, T* raw, int nx, int ny, long long pitch,
                          long long plane, int aos, cudaStream_t s) {
  unpack_kernel<T><<<grid_for((long long)nx * ny), 256, 0, s>>>(soa, raw, nx, ny, pitch, plane, aos);
  return cudaGetLastError();
}

template <typename T>
cudaError_t launch_set_ball(T* soa, int nx, int ny, long long pitch, long long plane, T hx, T hy,
                            T cx, T cy, T r, T s_val, cudaStream_t s) {
  set_ball_kernel<T><<<grid_for((long long)nx * ny), 256, 0, s>>>(soa, nx, ny, pitch, plane, hx,
                                                                  hy, cx, cy, r, s_val);
  return cudaGetLastError();
}

template <typename T>
cudaError_t launch_vtk_speed(const T* soa, int nx, int ny, long long pitch, long long plane,
                             unsigned* out, cudaStream_t s) {
  vtk_speed_kernel<T><<<grid_for((long long)nx * ny), 256, 0, s>>>(soa, nx, ny, pitch, plane, out);
  return cudaGetLastError();
}

#define LE2D_INST(T)                                                                             \
  template cudaError_t launch_pack<T>(const T*, T*, int, int, long long, long long, int,         \
                                      cudaStream_t);                                             \
  template cudaError_t launch_unpack<T>(const T*, T*, int, int, long long, long long, int,       \
                                        cudaStream_t);                                           \
  template cudaError_t launch_set_ball<T>(T*, int, int, long long, long long, T, T, T, T, T, T, \
                                          cudaStream_t);                                           \
  template cudaError_t launch_vtk_speed<T>(const T*, int, int, long long, long long, unsigned*,  \
                                           cudaStream_t);
LE2D_INST(float)
LE2D_INST(double)
#undef LE2D_INST

}  // namespace le2d
