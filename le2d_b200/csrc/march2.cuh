// Temporal blocking: two time steps per launch.  A warp marches its strip as in
// march.cuh, but every row that completes the first step (step A) is fed, still in
// registers, into a second x-sweep and y-pipeline (step B); only step B's rows are
// written.  The state is read once and written once per two steps.
//
// Halos.  A lane's x-sweep takes its neighbours' values by shuffles, so the lanes at the
// warp's edges see garbage there: step A is valid on the columns [xs+2, xs+32V-2) of the
// strip and step B, whose x-stencil reads step A's values two columns away, on
// [xs+4, xs+32V-4).  The strip therefore writes the lanes [H2, 32-H2), H2 = ceil(4 / V)
// (one lane for V = 4, two for V = 2).  In y, step B's rows [y0, y1) need step A's rows
// [y0-2, y1+2), which need the raw rows [y0-4, y1+4).
//
// Boundaries.  Step B must see step A's values exactly as a second single step would: at
// a column outside [0, nx) the value of the edge column (the reference clamps its
// indices), so edge strips overwrite step A's values there with the edge column's by
// warp shuffles; and at a row outside [0, ny) the edge row's, so the pseudo rows step A
// produces above row 0 / below row ny-1 are dropped and rows 0 / ny-1 are fed to step B
// once for every row of its stencil that they stand for.  (le_step_soa's far end is not a
// clamp; SoA tasks use single steps.)
#pragma once

#include "march.cuh"

namespace le2d {
namespace march {

template <typename T, int V, int NPF>
__host__ __device__ constexpr int warp_smem_elems2() {
  return (6 + NPF) * NF * 32 * V;  // input ring + step A ring + step B ring
}

// Columns of this lane outside [0, nx) take the values of column 0 / column nx-1, which
// the strip holds (lane (c - xs) / V, position (c - xs) % V).
template <typename T, int V>
__device__ __forceinline__ void clamp_columns(T (&v)[NF][V], int xs, int col0, int nx) {
  constexpr unsigned kAll = 0xffffffffu;
  const int lsrc = (-xs) / V, lpos = (-xs) % V;
  const int rsrc = (nx - 1 - xs) / V, rpos = (nx - 1 - xs) % V;
#pragma unroll
  for (int k = 0; k < NF; ++k) {
    const T lv = __shfl_sync(kAll, pick<T, V>(v[k], lpos < 0 ? 0 : lpos), lsrc & 31);
    const T rv = __shfl_sync(kAll, pick<T, V>(v[k], rpos < 0 ? 0 : rpos), rsrc & 31);
#pragma unroll
    for (int j = 0; j < V; ++j) {
      const int cc = col0 + j;
      v[k][j] = cc < 0 ? lv : (cc >= nx ? rv : v[k][j]);
    }
  }
}

// One x-swept row into a y-pipeline: store it in the ring slot, read it and the previous
// row back (aligned loads), advance the left-moving part.  `cy`: the y-sweep constants
// (Sweep, or YPairs for the FP32 pipeline).
template <typename T, int V, typename CY>
__device__ __forceinline__ void ring_left(YPipe<T, V>& yp, T (&f)[NF][V], T* ring, int slot,
                                          const CY& cy) {
  using VT = typename Vec<T, V>::type;
  constexpr int kIn = 32 * V;
  constexpr int kRow = NF * kIn;
  T* rs = ring + slot * kRow;
#pragma unroll
  for (int k = 0; k < NF; ++k) *reinterpret_cast<VT*>(rs + k * kIn) = pack(f[k]);
  const T* rp = ring + (slot == 0 ? 2 : slot - 1) * kRow;
  T cur[NF][V], pvy[V], psyy[V], pvx[V], psxy[V];
  unpack(*reinterpret_cast<const VT*>(rs + VY * kIn), cur[VY]);
  unpack(*reinterpret_cast<const VT*>(rs + SYY * kIn), cur[SYY]);
  unpack(*reinterpret_cast<const VT*>(rs + VX * kIn), cur[VX]);
  unpack(*reinterpret_cast<const VT*>(rs + SXY * kIn), cur[SXY]);
  unpack(*reinterpret_cast<const VT*>(rp + VY * kIn), pvy);
  unpack(*reinterpret_cast<const VT*>(rp + SYY * kIn), psyy);
  unpack(*reinterpret_cast<const VT*>(rp + VX * kIn), pvx);
  unpack(*reinterpret_cast<const VT*>(rp + SXY * kIn), psxy);
  yp.left(cur, pvy, psyy, pvx, psxy, cy);
}

// The row two above, completed: fields from the ring plus the pipeline's increments.
template <typename T, int V, typename CY>
__device__ __forceinline__ void ring_output(const YPipe<T, V>& yp, T (&out)[NF][V], const T* ring,
                                            int slot, const CY& cy) {
  using VT = typename Vec<T, V>::type;
  constexpr int kIn = 32 * V;
  constexpr int kRow = NF * kIn;
  const T* rg = ring + (slot == 2 ? 0 : slot + 1) * kRow;
#pragma unroll
  for (int k = 0; k < NF; ++k) unpack(*reinterpret_cast<const VT*>(rg + k * kIn), out[k]);
  yp.apply(out, cy);
}

// Advances one tile -- strip `strip`, rows [y0, y1) -- by two steps from g.src to g.dst.
// `smem_warp` = this warp's warp_smem_elems2() elements.  Called by all 32 lanes.
template <typename T, int V, int NPF, bool COHERENT>
__device__ __forceinline__ void march_tile2(const GridRef<T>& g, const StepConsts<T>& c, int strip,
                                            int y0, int y1, T* smem_warp) {
  using VT = typename Vec<T, V>::type;
  static_assert(NPF >= 2, "the input ring needs at least the current and the next row");
  constexpr int H2 = halo_lanes2(V);
  constexpr int kIn = 32 * V;
  constexpr int kOut = strip_cols2(V);
  constexpr int kRow = NF * kIn;
  const int lane = threadIdx.x & 31;
  T* in_ring = smem_warp + lane * V;
  T* a_ring = in_ring + NPF * kRow;
  T* b_ring = a_ring + 3 * kRow;
  const int xs = strip * kOut - H2 * V;
  const int col0 = xs + lane * V;
  const bool interior = xs >= 0 && xs + kIn <= g.nx;
  const bool writer = lane >= H2 && lane < 32 - H2 && col0 < g.nx;

  YPipe<T, V> ya, yb;
  ya.init();
  yb.init();
#pragma unroll
  for (int k = 0; k < NF; ++k) {
    *reinterpret_cast<VT*>(a_ring + 2 * kRow + k * kIn) = VT{};
    *reinterpret_cast<VT*>(b_ring + 2 * kRow + k * kIn) = VT{};
  }
#pragma unroll
  for (int j = 0; j < NPF - 1; ++j)
    fetch_row<T, V, COHERENT>(in_ring + j * kRow, g, source_row(y0 - 4 + j, g.ny, 0), col0, interior);
  int islot = 0, aslot = 0, bslot = 0;
  int bin = y0 - 2;  // step-B row index of the next row fed to step B
  for (int m = y0 - 4; m < y1 + 4; ++m) {
    {
      const int mm = m + NPF - 1;
      const int ns = islot + NPF - 1 >= NPF ? islot - 1 : islot + NPF - 1;
      if (mm < y1 + 4)
        fetch_row<T, V, COHERENT>(in_ring + ns * kRow, g, source_row(mm, g.ny, 0), col0, interior);
      else
        cp_async_commit();
    }
    cp_async_wait<NPF - 1>();
    T f[NF][V];
#pragma unroll
    for (int k = 0; k < NF; ++k)
      unpack(*reinterpret_cast<const VT*>(in_ring + islot * kRow + k * kIn), f[k]);
    if (!interior) clamp_lane<T, V>(f, col0, g.nx);
    sweep_x_lane<T, V>(f, c.x);
    ring_left(ya, f, a_ring, aslot, c.y);

    const int ka = m - 2;  // step-A row completed now
    // step B reads rows [y0-2, y1+2), clamped: row 0 stands for the rows above it and row
    // ny-1 for the rows below it
    int reps = 0;
    T ga[NF][V];
    if (m >= y0) {
      ring_output(ya, ga, a_ring, aslot, c.y);
      if (!interior) clamp_columns<T, V>(ga, xs, col0, g.nx);
      reps = ka < 0 || ka >= g.ny ? 0 : 1;
      if (ka == 0 && y0 < 2) reps += 2 - y0;
      if (ka == g.ny - 1 && y1 + 2 > g.ny) reps += y1 + 2 - g.ny;
    }
    ya.right(c.y);
    {
      for (int r = 0; r < reps; ++r) {
        T fb[NF][V];
#pragma unroll
        for (int k = 0; k < NF; ++k)
#pragma unroll
          for (int v = 0; v < V; ++v) fb[k][v] = ga[k][v];
        sweep_x_lane<T, V>(fb, c.x);
        ring_left(yb, fb, b_ring, bslot, c.y);
        if (bin >= y0 + 2) {  // step-B row bin-2 is complete
          T gb[NF][V];
          ring_output(yb, gb, b_ring, bslot, c.y);
          if (writer) {
            T* out = g.dst + (long long)(bin - 2) * g.pitch + col0;
#pragma unroll
            for (int k = 0; k < NF; ++k)
              if (in_dst(g, out + k * g.plane, V)) *reinterpret_cast<VT*>(out + k * g.plane) = pack(gb[k]);
          }
        }
        yb.right(c.y);
        bslot = bslot == 2 ? 0 : bslot + 1;
        ++bin;
      }
    }
    islot = islot + 1 == NPF ? 0 : islot + 1;
    aslot = aslot == 2 ? 0 : aslot + 1;
  }
}

}  // namespace march
}  // namespace le2d
