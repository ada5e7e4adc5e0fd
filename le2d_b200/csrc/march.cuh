// The strip-march body shared by the single-solve kernel (step_fused.cu) and the
// batched persistent kernel (batch.cu): one warp advances one tile -- a strip of
// 32*V columns by a segment of rows -- by one full time step (x-sweep then
// y-sweep, le2d simple/le_core.c:605-620).
//
// Per row the warp
//   1. loads the row's five fields (prefetched one row ahead),
//   2. x-sweeps the row in registers: each lane handles its V nodes, the
//      neighbouring invariants and face fluxes come from the adjacent lanes by
//      warp shuffles; the stencil reaches two nodes each way, so the outer lane
//      (two lanes when V = 1) on each side only supplies that halo,
//   3. keeps the x-swept row in a per-lane ring of three rows in shared memory,
//   4. feeds the row's y-invariants into a per-column y-pipeline held in registers
//      (face-form fluxes of the previous rows), which completes the y-sweep of the
//      row two above and writes it.
// A segment of L rows reads L+4 rows (two halo rows above and below).
#pragma once

#include "le2d_kernels.h"

namespace le2d {
namespace march {

template <typename T, int V>
struct Vec;
template <> struct Vec<float, 4> { using type = float4; };
template <> struct Vec<float, 2> { using type = float2; };
template <> struct Vec<double, 2> { using type = double2; };
template <> struct Vec<double, 1> { using type = double; };

__device__ __forceinline__ void unpack(const float4& a, float (&d)[4]) {
  d[0] = a.x; d[1] = a.y; d[2] = a.z; d[3] = a.w;
}
__device__ __forceinline__ void unpack(const float2& a, float (&d)[2]) { d[0] = a.x; d[1] = a.y; }
__device__ __forceinline__ void unpack(const double2& a, double (&d)[2]) { d[0] = a.x; d[1] = a.y; }
__device__ __forceinline__ void unpack(const double& a, double (&d)[1]) { d[0] = a; }
__device__ __forceinline__ float4 pack(const float (&d)[4]) { return make_float4(d[0], d[1], d[2], d[3]); }
__device__ __forceinline__ float2 pack(const float (&d)[2]) { return make_float2(d[0], d[1]); }
__device__ __forceinline__ double2 pack(const double (&d)[2]) { return make_double2(d[0], d[1]); }
__device__ __forceinline__ double pack(const double (&d)[1]) { return d[0]; }

// Loads of the state.  Read-only path (__ldg) when the state was written by an earlier
// launch; L2-only loads (ld.global.cg) when other warps of the same launch write it, as
// in the batched kernel, where the non-coherent L1 could hold stale lines.
template <bool COHERENT, typename VT>
__device__ __forceinline__ VT load_state(const VT* p) {
  if (COHERENT)
    return __ldcg(p);
  else
    return __ldg(p);
}

// A grid of one solve as the march sees it.
template <typename T>
struct GridRef {
  const T* src;
  T* dst;
  int nx, ny;
  long long pitch, plane;
  int far_rot;
};

// Optional receiver line: when `row` >= 0 and the march writes that row, vx and vy of
// the written columns also go to out[0 * pitch + i] and out[1 * pitch + i].
template <typename T>
struct RowTap {
  T* out;
  int row;
};

// Row index read for pipeline row m: clamped at the top; past the bottom either
// clamped (le_step) or the rows m-5 (le_step_soa's far end).
__device__ __forceinline__ int source_row(int m, int ny, int far_rot) {
  if (m < 0) return 0;
  if (m < ny) return m;
  return far_rot ? max(m - 5, 0) : ny - 1;
}

template <typename T, int V, bool COHERENT>
__device__ __forceinline__ void load_row(T (&f)[NF][V], const GridRef<T>& g, int row, int col0,
                                         bool interior) {
  using VT = typename Vec<T, V>::type;
  const T* base = g.src + (long long)row * g.pitch;
  if (interior) {
#pragma unroll
    for (int k = 0; k < NF; ++k)
      unpack(load_state<COHERENT>(reinterpret_cast<const VT*>(base + k * g.plane + col0)), f[k]);
  } else {
#pragma unroll
    for (int v = 0; v < V; ++v) {
      const int cc = min(max(col0 + v, 0), g.nx - 1);
#pragma unroll
      for (int k = 0; k < NF; ++k) f[k][v] = load_state<COHERENT>(base + k * g.plane + cc);
    }
  }
}

// x-sweep of the V nodes of this lane (row in registers, neighbours by shuffles).
// Face e (0..V) lies between node e-1 and node e of the lane; the neighbour lanes supply
// the fields of nodes -1 and V and the flux terms of their edge nodes.
template <typename T, int V>
__device__ __forceinline__ void sweep_x_lane(T (&f)[NF][V], const Sweep<T>& c) {
  constexpr unsigned kAll = 0xffffffffu;
  const T eps = tvd_eps<T>();
  // fields entering the x-invariants: vn = vx, sn = sxx, vt = vy, and sxy
  T lf[4], rf[4];
  {
    const int fk[4] = {VX, SXX, VY, SXY};
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      lf[q] = __shfl_up_sync(kAll, f[fk[q]][V - 1], 1);
      rf[q] = __shfl_down_sync(kAll, f[fk[q]][0], 1);
    }
  }
  T d[4][V + 1];
#pragma unroll
  for (int e = 0; e <= V; ++e) {
    const T nvx = e < V ? f[VX][e] : rf[0], pvx = e > 0 ? f[VX][e - 1] : lf[0];
    const T nsx = e < V ? f[SXX][e] : rf[1], psx = e > 0 ? f[SXX][e - 1] : lf[1];
    const T nvy = e < V ? f[VY][e] : rf[2], pvy = e > 0 ? f[VY][e - 1] : lf[2];
    const T nxy = e < V ? f[SXY][e] : rf[3], pxy = e > 0 ? f[SXY][e - 1] : lf[3];
    face_differences(nvx - pvx, nsx - psx, nvy - pvy, nxy - pxy, c, d[0][e], d[1][e], d[2][e],
                     d[3][e]);
  }
  T a[2][V], b[2][V];
#pragma unroll
  for (int q = 0; q < 2; ++q) {
    const T kc = q ? c.kc2 : c.kc1;
    {  // right-moving invariant (w1 / w3)
      const int k = 2 * q;
      T ps[V], t[V];
#pragma unroll
      for (int v = 0; v < V; ++v) {
        ps[v] = psi(ratio(d[k][v] + eps, d[k][v + 1] + eps), kc);
        t[v] = fma(ps[v], d[k][v + 1], -d[k][v + 1]);
      }
      const T t_in = __shfl_up_sync(kAll, t[V - 1], 1);
#pragma unroll
      for (int v = 0; v < V; ++v) a[q][v] = fma(-ps[v], d[k][v + 1], v ? t[v - 1] : t_in);
    }
    {  // left-moving invariant (w2 / w4)
      const int k = 2 * q + 1;
      T ps[V], h[V];
#pragma unroll
      for (int v = 0; v < V; ++v) {
        ps[v] = psi(ratio(eps - d[k][v + 1], eps - d[k][v]), kc);
        h[v] = fma(-ps[v], d[k][v], d[k][v]);
      }
      const T h_in = __shfl_down_sync(kAll, h[0], 1);
#pragma unroll
      for (int v = 0; v < V; ++v) b[q][v] = fma(ps[v], d[k][v], v < V - 1 ? h[v + 1] : h_in);
    }
  }
#pragma unroll
  for (int v = 0; v < V; ++v)
    apply_increment<0>(f[VX][v], f[VY][v], f[SXX][v], f[SXY][v], f[SYY][v], a[0][v], b[0][v],
                       a[1][v], b[1][v], c);
}

// Advances one tile -- strip `strip` (32*V columns, halo lanes included), rows [y0, y1) --
// by one step from g.src to g.dst.  `ring` = this warp's 3*NF*32*V elements of shared
// memory.  Called by all 32 lanes of a warp.
template <typename T, int V, int UNROLL, bool COHERENT, bool TAP>
__device__ __forceinline__ void march_tile(const GridRef<T>& g, const StepConsts<T>& c, int strip,
                                           int y0, int y1, T* ring_warp, const RowTap<T>& tap) {
  using VT = typename Vec<T, V>::type;
  constexpr int H = halo_lanes(V);
  constexpr int kIn = 32 * V;
  constexpr int kOut = strip_cols(V);
  const int lane = threadIdx.x & 31;
  T* ring = ring_warp + lane * V;
  const int xs = strip * kOut - H * V;
  const int col0 = xs + lane * V;
  const bool interior = xs >= 0 && xs + kIn <= g.nx;
  const bool writer = lane >= H && lane < 32 - H && col0 < g.nx;
  const T eps = tvd_eps<T>();
  const Sweep<T>& cy = c.y;

  // y-pipeline state per column (face j lies between rows j and j+1): the fields of row
  // m-1 that enter the y-invariants (vy, syy, vx, sxy); for w1/w3: P_{m-2}, t_{m-2} and
  // A_{m-1} (written out one row later); for w2/w4: Q_{m-2}, D_{m-2}, c_{m-2}.
  T pf[4][V], p2[2][V], t2[2][V], a2[2][V], q2[2][V], d2[2][V], c2[2][V];
#pragma unroll
  for (int v = 0; v < V; ++v) {
#pragma unroll
    for (int k = 0; k < 4; ++k) pf[k][v] = T(0);
#pragma unroll
    for (int q = 0; q < 2; ++q) p2[q][v] = t2[q][v] = a2[q][v] = q2[q][v] = d2[q][v] = c2[q][v] = T(0);
  }

  T nxt[NF][V];
  load_row<T, V, COHERENT>(nxt, g, source_row(y0 - 2, g.ny, g.far_rot), col0, interior);
  int slot = 0;  // ring slot of row m; row m-2 sits in (slot + 1) % 3
#pragma unroll UNROLL
  for (int m = y0 - 2; m < y1 + 2; ++m) {
    T f[NF][V];
#pragma unroll
    for (int k = 0; k < NF; ++k)
#pragma unroll
      for (int v = 0; v < V; ++v) f[k][v] = nxt[k][v];
    if (m + 1 < y1 + 2)
      load_row<T, V, COHERENT>(nxt, g, source_row(m + 1, g.ny, g.far_rot), col0, interior);

    sweep_x_lane<T, V>(f, c.x);

    T* rs = ring + slot * (NF * kIn);
#pragma unroll
    for (int k = 0; k < NF; ++k) *reinterpret_cast<VT*>(rs + k * kIn) = pack(f[k]);

    T a_out[2][V], b_out[2][V];
#pragma unroll
    for (int v = 0; v < V; ++v) {
      // D_{m-1} of the four invariants from the field differences of rows m-1 and m
      T d[4];
      face_differences(f[VY][v] - pf[0][v], f[SYY][v] - pf[1][v], f[VX][v] - pf[2][v],
                       f[SXY][v] - pf[3][v], cy, d[0], d[1], d[2], d[3]);
      pf[0][v] = f[VY][v];
      pf[1][v] = f[SYY][v];
      pf[2][v] = f[VX][v];
      pf[3][v] = f[SXY][v];
#pragma unroll
      for (int q = 0; q < 2; ++q) {
        const T kc = q ? cy.kc2 : cy.kc1;
        {  // right-moving: psi_{m-1}, A_{m-1} = t_{m-2} - psi_{m-1} D_{m-1}, t_{m-1}
          const T dd = d[2 * q];
          const T p1 = dd + eps;
          const T ps = psi(ratio(p2[q][v], p1), kc);
          a_out[q][v] = a2[q][v];
          a2[q][v] = fma(-ps, dd, t2[q][v]);
          t2[q][v] = fma(ps, dd, -dd);
          p2[q][v] = p1;
        }
        {  // left-moving: psi'_{m-1}, B_{m-2} = c_{m-2} - psi'_{m-1} D_{m-2}, c_{m-1}
          const T dd = d[2 * q + 1];
          const T q1 = eps - dd;
          const T ps = psi(ratio(q1, q2[q][v]), kc);
          b_out[q][v] = fma(-ps, d2[q][v], c2[q][v]);
          c2[q][v] = fma(ps, d2[q][v], dd);
          d2[q][v] = dd;
          q2[q][v] = q1;
        }
      }
    }

    if (m >= y0 + 2) {  // whole warp: halo lanes compute too, only the stores are predicated
      const int row = m - 2;
      const T* rg = ring + (slot == 2 ? 0 : slot + 1) * (NF * kIn);
      T gf[NF][V];
#pragma unroll
      for (int k = 0; k < NF; ++k) unpack(*reinterpret_cast<const VT*>(rg + k * kIn), gf[k]);
#pragma unroll
      for (int v = 0; v < V; ++v)
        apply_increment<1>(gf[VX][v], gf[VY][v], gf[SXX][v], gf[SXY][v], gf[SYY][v], a_out[0][v],
                           b_out[0][v], a_out[1][v], b_out[1][v], cy);
      if (writer) {
        T* out = g.dst + (long long)row * g.pitch + col0;
#pragma unroll
        for (int k = 0; k < NF; ++k) *reinterpret_cast<VT*>(out + k * g.plane) = pack(gf[k]);
        if (TAP && row == tap.row) {
          *reinterpret_cast<VT*>(tap.out + col0) = pack(gf[VX]);
          *reinterpret_cast<VT*>(tap.out + g.pitch + col0) = pack(gf[VY]);
        }
      }
    }
    slot = slot == 2 ? 0 : slot + 1;
  }
}

}  // namespace march
}  // namespace le2d
