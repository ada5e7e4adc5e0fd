// The plain scheme: one kernel per directional sweep, one thread per node, and the
// reference's per-node formula (tvd2 with its two slope ratios, le2d
// simple/le_core.c:48-69; reconstruct :251-257; inc_x / inc_y :221-249).  It
// reads the 5-node stencil of the five fields around each node and writes the
// node to a second buffer (Jacobi order).  Used as the "plain" comparator of the
// fused kernel and as an independent check of its face-form rearrangement.
#include "le2d_kernels.h"

namespace le2d {

namespace {

template <typename T>
__device__ __forceinline__ T superbee(T r) {
  return max3(T(0), fmin(T(1), r + r), fmin(T(2), r));
}

// tvd2 as the reference writes it, in T arithmetic with IEEE division.
template <typename T>
__device__ __forceinline__ T tvd2(T c, T u_2, T u_1, T u, T u1) {
  const T eps = tvd_eps<T>();
  T r1 = u - u_1;
  T r2 = u1 - u;
  r1 += eps;
  r2 += eps;
  const T r = r1 / r2;
  r1 = u_1 - u_2;
  r2 = u - u_1;
  r1 += eps;
  r2 += eps;
  const T r_1 = r1 / r2;
  const T f12 = u + superbee(r) / T(2) * (T(1) - c) * (u1 - u);
  const T f_12 = u_1 + superbee(r_1) / T(2) * (T(1) - c) * (u - u_1);
  return u - c * (f12 - f_12);
}

// FP64: le_min / le_max / le_max3 (simple/le_core.c:31-33) as written, so NaN and signed
// zeros come out as in the reference.
__device__ __forceinline__ double ref_min(double a, double b) { return a > b ? b : a; }
__device__ __forceinline__ double ref_max(double a, double b) { return a > b ? a : b; }

// FP64 tvd2 operation by operation in uncontracted arithmetic, with IEEE division: the
// reference double build's result bit for bit.
template <>
__device__ __forceinline__ double tvd2<double>(double c, double u_2, double u_1, double u, double u1) {
  using namespace ex;
  const double eps = tvd_eps<double>();
  const double r = add(sub(u, u_1), eps) / add(sub(u1, u), eps);
  const double r_1 = add(sub(u_1, u_2), eps) / add(sub(u, u_1), eps);
  const double hc = mul(0.5, sub(1.0, c));  // (1 - c) / 2: halving is exact
  const double s = ref_max(0.0, ref_max(ref_min(1.0, r + r), ref_min(2.0, r)));
  const double s_1 = ref_max(0.0, ref_max(ref_min(1.0, r_1 + r_1), ref_min(2.0, r_1)));
  const double f12 = add(u, mul(mul(s, hc), sub(u1, u)));
  const double f_12 = add(u_1, mul(mul(s_1, hc), sub(u, u_1)));
  return sub(u, mul(c, sub(f12, f_12)));
}

// Index of stencil node q along a line of n nodes: clamped, or (far_rot, y only) the
// rows n-5, n-4 past the end as le_step_soa sees them.
__device__ __forceinline__ int line_index(int q, int n, int far_rot) {
  if (q < 0) return 0;
  if (q < n) return q;
  return far_rot ? max(q - 5, 0) : n - 1;
}

template <typename T, int AXIS>
__global__ void sweep_plain_kernel(const T* __restrict__ src, T* __restrict__ dst, int nx, int ny,
                                   long long pitch, long long plane, Sweep<T> c, T k1, T k2,
                                   int far_rot) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  if (i >= nx || j >= ny) return;
  const int n = AXIS == 0 ? nx : ny;
  const int pos = AXIS == 0 ? i : j;
  T w[5][4];
  T node[NF];
#pragma unroll
  for (int o = -2; o <= 2; ++o) {
    const int q = line_index(pos + o, n, AXIS == 1 ? far_rot : 0);
    const int ii = AXIS == 0 ? q : i;
    const int jj = AXIS == 0 ? j : q;
    const T* b = src + (long long)jj * pitch + ii;
    T fv[NF];
#pragma unroll
    for (int k = 0; k < NF; ++k) fv[k] = b[k * plane];
    if constexpr (sizeof(T) == 8) {
      const T vn = AXIS == 0 ? fv[VX] : fv[VY], vt = AXIS == 0 ? fv[VY] : fv[VX];
      const T sn = AXIS == 0 ? fv[SXX] : fv[SYY];
      ex::invariants(vn, sn, vt, fv[SXY], c, w[o + 2]);
    } else {
      omega<AXIS>(fv[VX], fv[VY], fv[SXX], fv[SXY], fv[SYY], c, w[o + 2][0], w[o + 2][1],
                  w[o + 2][2], w[o + 2][3]);
    }
    if (o == 0)
#pragma unroll
      for (int k = 0; k < NF; ++k) node[k] = fv[k];
  }
  // reconstruct (simple/le_core.c:251-257): the change of each invariant
  const T c1 = tvd2(k1, w[0][0], w[1][0], w[2][0], w[3][0]) - w[2][0];
  const T c2 = tvd2(k1, w[4][1], w[3][1], w[2][1], w[1][1]) - w[2][1];
  const T c3 = tvd2(k2, w[0][2], w[1][2], w[2][2], w[3][2]) - w[2][2];
  const T c4 = tvd2(k2, w[4][3], w[3][3], w[2][3], w[1][3]) - w[2][3];
  if constexpr (sizeof(T) == 8) {
    ex::increment<AXIS>(node[VX], node[VY], node[SXX], node[SXY], node[SYY], c1, c2, c3, c4, c);
  } else {
    // inc_x / inc_y (simple/le_core.c:221-249)
    const T d1 = T(0.5) * c1, d2 = T(0.5) * c2, d3 = T(0.5) * c3, d4 = T(0.5) * c4;
    T& vn = AXIS == 0 ? node[VX] : node[VY];
    T& vt = AXIS == 0 ? node[VY] : node[VX];
    T& sn = AXIS == 0 ? node[SXX] : node[SYY];
    T& so = AXIS == 0 ? node[SYY] : node[SXX];
    vn += d1 + d2;
    vt += d3 + d4;
    sn += (d2 - d1) * c.rhoc1;
    so += (d2 - d1) * c.rhoc3;
    node[SXY] += c.rhoc2 * (d4 - d3);
  }
  T* o = dst + (long long)j * pitch + i;
#pragma unroll
  for (int k = 0; k < NF; ++k) o[k * plane] = node[k];
}

}  // namespace

template <typename T>
cudaError_t launch_split_sweep(int axis, const T* src, T* dst, int nx, int ny, long long pitch,
                               long long plane, const Sweep<T>& c, T k1, T k2, int far_rot,
                               cudaStream_t s) {
  const dim3 block(32, 8);
  const dim3 grid((nx + 31) / 32, (ny + 7) / 8);
  if (axis == 0)
    sweep_plain_kernel<T, 0><<<grid, block, 0, s>>>(src, dst, nx, ny, pitch, plane, c, k1, k2, 0);
  else
    sweep_plain_kernel<T, 1><<<grid, block, 0, s>>>(src, dst, nx, ny, pitch, plane, c, k1, k2,
                                                    far_rot);
  return cudaGetLastError();
}

template cudaError_t launch_split_sweep<float>(int, const float*, float*, int, int, long long,
                                               long long, const Sweep<float>&, float, float, int,
                                               cudaStream_t);
template cudaError_t launch_split_sweep<double>(int, const double*, double*, int, int, long long,
                                                long long, const Sweep<double>&, double, double,
                                                int, cudaStream_t);

}  // namespace le2d
