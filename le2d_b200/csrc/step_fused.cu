// Fused time step: x-sweep and y-sweep in one kernel, one read and one write of
// the state per step (le2d simple/le_core.c:605-620: le_step = le_step_x then
// le_step_y, both with Jacobi semantics and clamped ends).
//
// Decomposition ("strip march").  Each warp owns a vertical strip of 32*V
// columns (V = 16 bytes / sizeof(T): 4 floats or 2 doubles per lane, one 128-bit
// access per field) and walks down a segment of rows.  For every row it
//   1. loads the row's five fields (prefetched one row ahead),
//   2. x-sweeps the row in registers: each lane handles its V nodes, the
//      neighbouring invariants and face fluxes come from the adjacent lanes by
//      warp shuffles; lanes 0 and 31 only supply that halo, so a strip outputs
//      30*V columns and adjacent strips overlap by 2*V columns,
//   3. keeps the x-swept row in a per-lane ring of three rows in shared memory,
//   4. feeds the row's y-invariants into a per-column y-pipeline held in
//      registers (face-form fluxes of the previous rows), which completes the
//      y-sweep of the row two above and writes it.
// A segment of L rows reads L+4 rows (two halo rows above and below), so the
// state is read about (1 + 4/L)(32/30) times and written once per step.
#include "le2d_kernels.h"

namespace le2d {

namespace {

template <typename T>
struct FusedParams {
  const T* __restrict__ src;
  T* __restrict__ dst;
  int nx, ny;
  long long pitch, plane;
  int nstrips, seg_len, ntasks;
  int far_rot;
  StepConsts<T> c;
};

constexpr int kWarps = 4;  // warps per block; warps are independent

template <typename T, int V>
struct Vec;
template <>
struct Vec<float, 4> {
  using type = float4;
};
template <>
struct Vec<double, 2> {
  using type = double2;
};

__device__ __forceinline__ void unpack(const float4& a, float (&d)[4]) {
  d[0] = a.x; d[1] = a.y; d[2] = a.z; d[3] = a.w;
}
__device__ __forceinline__ void unpack(const double2& a, double (&d)[2]) {
  d[0] = a.x; d[1] = a.y;
}
__device__ __forceinline__ float4 pack(const float (&d)[4]) { return make_float4(d[0], d[1], d[2], d[3]); }
__device__ __forceinline__ double2 pack(const double (&d)[2]) { return make_double2(d[0], d[1]); }

// Row index read for pipeline row m: clamped at the top; past the bottom either
// clamped (le_step) or the rows m-5 (le_step_soa, see the oracle's o_sweep_line).
__device__ __forceinline__ int source_row(int m, int ny, int far_rot) {
  if (m < 0) return 0;
  if (m < ny) return m;
  return far_rot ? max(m - 5, 0) : ny - 1;
}

template <typename T, int V>
__device__ __forceinline__ void load_row(T (&f)[NF][V], const FusedParams<T>& p, int row, int col0,
                                         bool interior) {
  using VT = typename Vec<T, V>::type;
  const T* base = p.src + (long long)row * p.pitch;
  if (interior) {
#pragma unroll
    for (int k = 0; k < NF; ++k)
      unpack(__ldg(reinterpret_cast<const VT*>(base + k * p.plane + col0)), f[k]);
  } else {
#pragma unroll
    for (int v = 0; v < V; ++v) {
      const int cc = min(max(col0 + v, 0), p.nx - 1);
#pragma unroll
      for (int k = 0; k < NF; ++k) f[k][v] = __ldg(base + k * p.plane + cc);
    }
  }
}

// x-sweep of the V nodes of this lane (row in registers, neighbours by shuffles).
template <typename T, int V>
__device__ __forceinline__ void sweep_x_lane(T (&f)[NF][V], const Sweep<T>& c) {
  constexpr unsigned kAll = 0xffffffffu;
  const T eps = tvd_eps<T>();
  T w[4][V];
#pragma unroll
  for (int v = 0; v < V; ++v)
    omega<0>(f[VX][v], f[VY][v], f[SXX][v], f[SXY][v], f[SYY][v], c, w[0][v], w[1][v], w[2][v],
             w[3][v]);
  T a[2][V], b[2][V];
#pragma unroll
  for (int q = 0; q < 2; ++q) {
    const T kc = q ? c.kc2 : c.kc1;
    // right-moving invariant (w1 / w3): faces e = 0..V, face e sits left of node v = e
    {
      const int k = 2 * q;
      const T left = __shfl_up_sync(kAll, w[k][V - 1], 1);
      const T right = __shfl_down_sync(kAll, w[k][0], 1);
      T d[V + 1], pp[V + 1];
      d[0] = w[k][0] - left;
#pragma unroll
      for (int e = 1; e < V; ++e) d[e] = w[k][e] - w[k][e - 1];
      d[V] = right - w[k][V - 1];
#pragma unroll
      for (int e = 0; e <= V; ++e) pp[e] = d[e] + eps;
      T fl[V];
#pragma unroll
      for (int v = 0; v < V; ++v) fl[v] = flux_fwd(w[k][v], pp[v], pp[v + 1], d[v + 1], kc);
      const T f_in = __shfl_up_sync(kAll, fl[V - 1], 1);
#pragma unroll
      for (int v = 0; v < V; ++v) a[q][v] = (v ? fl[v - 1] : f_in) - fl[v];
    }
    // left-moving invariant (w2 / w4)
    {
      const int k = 2 * q + 1;
      const T left = __shfl_up_sync(kAll, w[k][V - 1], 1);
      const T right = __shfl_down_sync(kAll, w[k][0], 1);
      T d[V + 1], qq[V + 1];
      d[0] = w[k][0] - left;
#pragma unroll
      for (int e = 1; e < V; ++e) d[e] = w[k][e] - w[k][e - 1];
      d[V] = right - w[k][V - 1];
#pragma unroll
      for (int e = 0; e <= V; ++e) qq[e] = eps - d[e];
      T gl[V];
#pragma unroll
      for (int v = 0; v < V; ++v) gl[v] = flux_bwd(w[k][v], qq[v], qq[v + 1], d[v], kc);
      const T g_in = __shfl_down_sync(kAll, gl[0], 1);
#pragma unroll
      for (int v = 0; v < V; ++v) b[q][v] = (v < V - 1 ? gl[v + 1] : g_in) - gl[v];
    }
  }
#pragma unroll
  for (int v = 0; v < V; ++v)
    apply_increment<0>(f[VX][v], f[VY][v], f[SXX][v], f[SXY][v], f[SYY][v], a[0][v], b[0][v],
                       a[1][v], b[1][v], c);
}

template <typename T, int V>
__global__ void __launch_bounds__(kWarps * 32) fused_step_kernel(const FusedParams<T> p) {
  using VT = typename Vec<T, V>::type;
  constexpr int kIn = 32 * V;   // columns held by a warp
  constexpr int kOut = 30 * V;  // columns written by a warp
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int lane = threadIdx.x & 31;
  const int wib = threadIdx.x >> 5;
  const int task = blockIdx.x * kWarps + wib;
  if (task >= p.ntasks) return;  // whole warp leaves together
  T* ring = reinterpret_cast<T*>(smem_raw) + wib * (3 * NF * kIn) + lane * V;

  const int strip = task % p.nstrips;
  const int seg = task / p.nstrips;
  const int xs = strip * kOut - V;
  const int col0 = xs + lane * V;
  const bool interior = xs >= 0 && xs + kIn <= p.nx;
  const bool writer = lane >= 1 && lane <= 30 && col0 < p.nx;
  const int y0 = seg * p.seg_len;
  const int y1 = min(y0 + p.seg_len, p.ny);
  const T eps = tvd_eps<T>();
  const Sweep<T>& cy = p.c.y;

  // y-pipeline state per column: u_{m-1} (4 invariants); for w1/w3: P_{m-2}, F_{m-2},
  // A_{m-2} = F_{m-3} - F_{m-2}; for w2/w4: Q_{m-2}, D_{m-2}, G_{m-2}.
  T um1[4][V], p2[2][V], f2[2][V], a2[2][V], q2[2][V], d2[2][V], g2[2][V];
#pragma unroll
  for (int v = 0; v < V; ++v) {
#pragma unroll
    for (int k = 0; k < 4; ++k) um1[k][v] = T(0);
#pragma unroll
    for (int q = 0; q < 2; ++q) p2[q][v] = f2[q][v] = a2[q][v] = q2[q][v] = d2[q][v] = g2[q][v] = T(0);
  }

  T nxt[NF][V];
  load_row<T, V>(nxt, p, source_row(y0 - 2, p.ny, p.far_rot), col0, interior);
  int slot = 0;  // ring slot of row m; row m-2 sits in (slot + 1) % 3
  for (int m = y0 - 2; m < y1 + 2; ++m) {
    T f[NF][V];
#pragma unroll
    for (int k = 0; k < NF; ++k)
#pragma unroll
      for (int v = 0; v < V; ++v) f[k][v] = nxt[k][v];
    if (m + 1 < y1 + 2) load_row<T, V>(nxt, p, source_row(m + 1, p.ny, p.far_rot), col0, interior);

    sweep_x_lane<T, V>(f, p.c.x);

    T* rs = ring + slot * (NF * kIn);
#pragma unroll
    for (int k = 0; k < NF; ++k) *reinterpret_cast<VT*>(rs + k * kIn) = pack(f[k]);

    T a_out[2][V], b_out[2][V];
#pragma unroll
    for (int v = 0; v < V; ++v) {
      T u[4];
      omega<1>(f[VX][v], f[VY][v], f[SXX][v], f[SXY][v], f[SYY][v], cy, u[0], u[1], u[2], u[3]);
#pragma unroll
      for (int q = 0; q < 2; ++q) {
        const T kc = q ? cy.kc2 : cy.kc1;
        {  // right-moving: F_{m-1}, A_{m-1}
          const int k = 2 * q;
          const T d1 = u[k] - um1[k][v];
          const T p1 = d1 + eps;
          const T f1 = flux_fwd(um1[k][v], p2[q][v], p1, d1, kc);
          a_out[q][v] = a2[q][v];
          a2[q][v] = f2[q][v] - f1;
          f2[q][v] = f1;
          p2[q][v] = p1;
          um1[k][v] = u[k];
        }
        {  // left-moving: G_{m-1}, B_{m-2}
          const int k = 2 * q + 1;
          const T d1 = u[k] - um1[k][v];
          const T q1 = eps - d1;
          const T g1 = flux_bwd(um1[k][v], q2[q][v], q1, d2[q][v], kc);
          b_out[q][v] = g1 - g2[q][v];
          g2[q][v] = g1;
          q2[q][v] = q1;
          d2[q][v] = d1;
          um1[k][v] = u[k];
        }
      }
    }

    if (m >= y0 + 2 && writer) {
      const int row = m - 2;
      const T* rg = ring + (slot == 2 ? 0 : slot + 1) * (NF * kIn);
      T g[NF][V];
#pragma unroll
      for (int k = 0; k < NF; ++k) unpack(*reinterpret_cast<const VT*>(rg + k * kIn), g[k]);
#pragma unroll
      for (int v = 0; v < V; ++v)
        apply_increment<1>(g[VX][v], g[VY][v], g[SXX][v], g[SXY][v], g[SYY][v], a_out[0][v],
                           b_out[0][v], a_out[1][v], b_out[1][v], cy);
      T* out = p.dst + (long long)row * p.pitch + col0;
#pragma unroll
      for (int k = 0; k < NF; ++k) *reinterpret_cast<VT*>(out + k * p.plane) = pack(g[k]);
    }
    slot = slot == 2 ? 0 : slot + 1;
  }
}

}  // namespace

template <typename T>
int fused_resident_warps(int device) {
  constexpr int V = 16 / (int)sizeof(T);
  int sms = 0, per_sm = 0;
  if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device) != cudaSuccess) return 0;
  const size_t smem = (size_t)kWarps * 3 * NF * 32 * V * sizeof(T);
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fused_step_kernel<T, V>, kWarps * 32,
                                                    smem) != cudaSuccess)
    return 0;
  return sms * per_sm * kWarps;
}

template <typename T>
FusedPlan plan_fused(int nx, int ny, int resident_warps, int min_seg) {
  constexpr int V = 16 / (int)sizeof(T);
  FusedPlan pl;
  pl.nstrips = (nx + strip_out<T>() - 1) / strip_out<T>();
  int target = resident_warps > 0 ? resident_warps / pl.nstrips : 1;
  if (target < 1) target = 1;
  int seg = (ny + target - 1) / target;
  if (seg < min_seg) seg = min_seg;
  if (seg > ny) seg = ny;
  pl.seg_len = seg;
  pl.nsegs = (ny + seg - 1) / seg;
  pl.ntasks = pl.nstrips * pl.nsegs;
  pl.threads = kWarps * 32;
  pl.blocks = (pl.ntasks + kWarps - 1) / kWarps;
  pl.smem = (size_t)kWarps * 3 * NF * 32 * V * sizeof(T);
  return pl;
}

template <typename T>
cudaError_t launch_fused_step(const T* src, T* dst, int nx, int ny, long long pitch,
                              long long plane, const StepConsts<T>& c, int far_rot,
                              const FusedPlan& plan, cudaStream_t s) {
  constexpr int V = 16 / (int)sizeof(T);
  FusedParams<T> p;
  p.src = src;
  p.dst = dst;
  p.nx = nx;
  p.ny = ny;
  p.pitch = pitch;
  p.plane = plane;
  p.nstrips = plan.nstrips;
  p.seg_len = plan.seg_len;
  p.ntasks = plan.ntasks;
  p.far_rot = far_rot;
  p.c = c;
  fused_step_kernel<T, V><<<plan.blocks, plan.threads, plan.smem, s>>>(p);
  return cudaGetLastError();
}

#define LE2D_INST(T)                                                                            \
  template int fused_resident_warps<T>(int);                                                    \
  template FusedPlan plan_fused<T>(int, int, int, int);                                         \
  template cudaError_t launch_fused_step<T>(const T*, T*, int, int, long long, long long,       \
                                            const StepConsts<T>&, int, const FusedPlan&,        \
                                            cudaStream_t);
LE2D_INST(float)
LE2D_INST(double)
#undef LE2D_INST

}  // namespace le2d
