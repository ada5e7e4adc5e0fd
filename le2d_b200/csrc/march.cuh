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

// Bounds-checked build (-DLE2D_CHECK, the library under lib/checked/): every access of the
// state checks that it stays inside the five planes of the buffer it addresses -- row in
// [0, ny), columns in [0, pitch) -- and counts it in g_check_violations and skips it (a load
// reads 0) when it does not, so a wrong index is reported without touching memory outside
// the buffer.  In the normal build the checks are constant true and vanish.  Each
// translation unit that marches tiles has its own counter; check_violations() in that unit
// reads and clears it.
#ifdef LE2D_CHECK
static __device__ unsigned long long g_check_violations = 0;
#endif

template <typename T>
__device__ __forceinline__ bool in_grid(const T* base, const T* p, long long pitch, long long plane,
                                        int ny, int ncols) {
#ifdef LE2D_CHECK
  const long long off = p - base;
  bool ok = off >= 0 && off < 5 * plane;
  if (ok) {
    const long long q = off % plane;
    ok = q / pitch < ny && q % pitch + ncols <= pitch;
  }
  if (!ok) atomicAdd(&g_check_violations, 1ULL);
  return ok;
#else
  return true;
#endif
}
template <typename T>
__device__ __forceinline__ bool in_src_checked(const GridRef<T>& g, const T* p, int ncols) {
  return in_grid(g.src, p, g.pitch, g.plane, g.ny, ncols);
}
template <typename T>
__device__ __forceinline__ bool in_dst_checked(const GridRef<T>& g, const T* p, int ncols) {
  return in_grid<T>(g.dst, p, g.pitch, g.plane, g.ny, ncols);
}
// A receiver line: two rows (vx, vy) of `pitch` elements per sample.
__device__ __forceinline__ bool in_line_checked(int col0, int ncols, long long pitch) {
#ifdef LE2D_CHECK
  const bool ok = col0 >= 0 && col0 + ncols <= pitch;
  if (!ok) atomicAdd(&g_check_violations, 1ULL);
  return ok;
#else
  return true;
#endif
}
// The checks as they appear at the accesses: the literal `true` in the normal build, so its
// code is exactly the unchecked code.
#ifdef LE2D_CHECK
#define in_src(g, p, n) in_src_checked(g, p, n)
#define in_dst(g, p, n) in_dst_checked(g, p, n)
#define in_line(c, n, pitch) in_line_checked(c, n, pitch)
#else
#define in_src(g, p, n) true
#define in_dst(g, p, n) true
#define in_line(c, n, pitch) true
#endif

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

// FP64 x-sweep in the reference's flux form (tvd2, simple/le_core.c:48-69): invariants
// w of each node, face differences D = w_{i+1} - w_i, slope ratios, limited fluxes
// F_i = w_i + psi_i D_i (right-moving w1, w3) and G_i = w_i - psi'_i D_{i-1} (left-moving
// w2, w4), then u - k (f12 - f_12) - u and inc_x, every operation rounded as the reference
// rounds it, so the result is the reference double build's bit for bit (up to the sign of
// zero and the division's rounding, see ratio(double)).  Face e (0..V) of the lane lies
// between its nodes e-1 and e; the neighbour lanes supply the invariants of nodes -1 and V
// and the fluxes of their edge nodes.
template <int V>
__device__ __forceinline__ void sweep_x_lane_exact(double (&f)[NF][V], const Sweep<double>& c) {
  constexpr unsigned kAll = 0xffffffffu;
  const double eps = tvd_eps<double>();
  double w[4][V + 2];  // nodes -1 .. V
#pragma unroll
  for (int v = 0; v < V; ++v) {
    double wv[4];
    ex::invariants(f[VX][v], f[SXX][v], f[VY][v], f[SXY][v], c, wv);
#pragma unroll
    for (int k = 0; k < 4; ++k) w[k][v + 1] = wv[k];
  }
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    w[k][0] = __shfl_up_sync(kAll, w[k][V], 1);
    w[k][V + 1] = __shfl_down_sync(kAll, w[k][1], 1);
  }
  double dw[4][V];
#pragma unroll
  for (int q = 0; q < 2; ++q) {
    const double kc = q ? c.kc2 : c.kc1;
    const double kk = q ? c.k2 : c.k1;
    {  // right-moving invariant (w1 / w3): psi_v = psi(P_left / P_right), F_v
      const int k = 2 * q;
      double d[V + 1], fl[V];
#pragma unroll
      for (int e = 0; e <= V; ++e) d[e] = ex::sub(w[k][e + 1], w[k][e]);
#pragma unroll
      for (int v = 0; v < V; ++v) {
        const double ps = psi_ratio(ex::add(d[v], eps), ex::add(d[v + 1], eps), kc);
        fl[v] = ex::add(w[k][v + 1], ex::mul(ps, d[v + 1]));
      }
      const double f_in = __shfl_up_sync(kAll, fl[V - 1], 1);
#pragma unroll
      for (int v = 0; v < V; ++v) dw[k][v] = ex::change(w[k][v + 1], kk, ex::sub(fl[v], v ? fl[v - 1] : f_in));
    }
    {  // left-moving invariant (w2 / w4): psi'_v = psi(Q_right / Q_left), G_v
      const int k = 2 * q + 1;
      double d[V + 1], gl[V];
#pragma unroll
      for (int e = 0; e <= V; ++e) d[e] = ex::sub(w[k][e + 1], w[k][e]);
#pragma unroll
      for (int v = 0; v < V; ++v) {
        const double ps = psi_ratio(ex::sub(eps, d[v + 1]), ex::sub(eps, d[v]), kc);
        gl[v] = ex::sub(w[k][v + 1], ex::mul(ps, d[v]));
      }
      const double g_in = __shfl_down_sync(kAll, gl[0], 1);
#pragma unroll
      for (int v = 0; v < V; ++v)
        dw[k][v] = ex::change(w[k][v + 1], kk, ex::sub(gl[v], v < V - 1 ? gl[v + 1] : g_in));
    }
  }
#pragma unroll
  for (int v = 0; v < V; ++v)
    ex::increment<0>(f[VX][v], f[VY][v], f[SXX][v], f[SXY][v], f[SYY][v], dw[0][v], dw[1][v],
                     dw[2][v], dw[3][v], c);
}

// FP32 x-sweep of the V nodes of this lane in the difference form, one invariant at a time
// (row in registers, neighbours by shuffles).  Face e (0..V) lies between node e-1 and
// node e of the lane; the neighbour lanes supply the fields of nodes -1 and V and the flux
// terms of their edge nodes.
template <typename T, int V>
__device__ __forceinline__ void sweep_x_lane_diff(T (&f)[NF][V], const Sweep<T>& c) {
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
        ps[v] = psi_ratio(d[k][v] + eps, d[k][v + 1] + eps, kc);
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
        ps[v] = psi_ratio(eps - d[k][v + 1], eps - d[k][v], kc);
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

// Packed FP32 arithmetic (f32x2: two independent lanes of the same operation, each
// rounded as its scalar form).
__device__ __forceinline__ float2 f2(float a, float b) { return make_float2(a, b); }
__device__ __forceinline__ float2 add2(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 mul2(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 fma2(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
__device__ __forceinline__ float2 superbee2(float2 r) {
  return f2(fmaxf(__saturatef(r.x + r.x), fminf(2.0f, r.x)),
            fmaxf(__saturatef(r.y + r.y), fminf(2.0f, r.y)));
}
__device__ __forceinline__ float2 ratio2(float2 a, float2 b) {
  float x, y;
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(x) : "f"(b.x));
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(b.y));
  return mul2(a, f2(x, y));
}

// FP32 x-sweep of the V nodes of this lane in the difference form (row in registers,
// neighbours by shuffles), on pairs of invariants: (w1, w3) move right and (w2, w4) left,
// and the two of a pair go through the same operations with their own constants, so each
// pair runs as packed f32x2 arithmetic -- the field differences of a face are formed as
// (dvx, dvy) and (dsxx, dsxy), which give (D1, D3) and (D2, D4) in one packed FMA each.
// Every element sees the operations of sweep_x_lane_diff in the same order; signs are
// arranged as in the packed y-pipeline, the right-moving pair keeping -t and -A, so no
// negation is needed.  The two forms give the same bits: t, A, -t and -A are never -0 (an
// exact zero of a rounded sum is +0, and psi >= 0), so where A = +0 the sums A + B and
// B - A that enter the fields are B + 0 in both.  About 9 % fewer instructions per
// node-update in the fused kernels; the batched kernel, at a different occupancy, runs
// the scalar form faster.  Face e (0..V) lies between node e-1 and node e of the lane;
// the neighbour lanes supply the fields of nodes -1 and V and the flux terms of their edge
// nodes.
template <int V>
__device__ __forceinline__ void sweep_x_lane_packed(float (&f)[NF][V], const Sweep<float>& c) {
  constexpr unsigned kAll = 0xffffffffu;
  const float2 m1 = f2(-1.f, -1.f), eps = f2(1e-6f, 1e-6f);
  // fields entering the x-invariants: vn = vx, sn = sxx, vt = vy, and sxy
  float lf[4], rf[4];
  {
    const int fk[4] = {VX, SXX, VY, SXY};
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      lf[q] = __shfl_up_sync(kAll, f[fk[q]][V - 1], 1);
      rf[q] = __shfl_down_sync(kAll, f[fk[q]][0], 1);
    }
  }
  float2 dr[V + 1], dl[V + 1];  // (D1, D3) and (D2, D4) of face e
#pragma unroll
  for (int e = 0; e <= V; ++e) {
    const float nvx = e < V ? f[VX][e] : rf[0], pvx = e > 0 ? f[VX][e - 1] : lf[0];
    const float nsx = e < V ? f[SXX][e] : rf[1], psx = e > 0 ? f[SXX][e - 1] : lf[1];
    const float nvy = e < V ? f[VY][e] : rf[2], pvy = e > 0 ? f[VY][e - 1] : lf[2];
    const float nxy = e < V ? f[SXY][e] : rf[3], pxy = e > 0 ? f[SXY][e - 1] : lf[3];
    const float2 dv = f2(nvx - pvx, nvy - pvy);
    const float2 ds = f2(nsx - psx, nxy - pxy);
    dr[e] = fma2(ds, c.nirp, dv);
    dl[e] = fma2(ds, c.irp, dv);
  }
  float2 na[V], b[V];  // (-A1, -A3) and (B2, B4) of node v
  {  // right-moving (w1, w3): psi_v = psi(P_v / P_{v+1}), -t_v = D_{v+1} - psi_v D_{v+1}
    float2 p[V + 1], ps[V], nt[V];
#pragma unroll
    for (int e = 0; e <= V; ++e) p[e] = add2(dr[e], eps);
#pragma unroll
    for (int v = 0; v < V; ++v) {
      const float2 phi = superbee2(ratio2(p[v], p[v + 1]));
      ps[v] = mul2(c.kcp, phi);
      nt[v] = fma2(mul2(c.nkcp, phi), dr[v + 1], dr[v + 1]);
    }
    const float2 nt_in = f2(__shfl_up_sync(kAll, nt[V - 1].x, 1), __shfl_up_sync(kAll, nt[V - 1].y, 1));
#pragma unroll
    for (int v = 0; v < V; ++v) na[v] = fma2(ps[v], dr[v + 1], v ? nt[v - 1] : nt_in);
  }
  {  // left-moving (w2, w4): psi'_v = psi(Q_{v+1} / Q_v), h_v = D_v - psi'_v D_v
    float2 q[V + 1], ps[V], h[V];
#pragma unroll
    for (int e = 0; e <= V; ++e) q[e] = fma2(dl[e], m1, eps);  // eps - D
#pragma unroll
    for (int v = 0; v < V; ++v) {
      const float2 phi = superbee2(ratio2(q[v + 1], q[v]));
      ps[v] = mul2(c.kcp, phi);
      h[v] = fma2(mul2(c.nkcp, phi), dl[v], dl[v]);
    }
    const float2 h_in = f2(__shfl_down_sync(kAll, h[0].x, 1), __shfl_down_sync(kAll, h[0].y, 1));
#pragma unroll
    for (int v = 0; v < V; ++v) b[v] = fma2(ps[v], dl[v], v < V - 1 ? h[v + 1] : h_in);
  }
#pragma unroll
  for (int v = 0; v < V; ++v) {  // apply_increment<0>
    const float2 sum = fma2(na[v], m1, b[v]);  // (A1 + B2, A3 + B4)
    const float2 dif = add2(b[v], na[v]);      // (B2 - A1, B4 - A3)
    f[VX][v] = fmaf(c.hk1, sum.x, f[VX][v]);
    f[VY][v] = fmaf(c.hk2, sum.y, f[VY][v]);
    f[SXX][v] = fmaf(c.hk1rc1, dif.x, f[SXX][v]);
    f[SYY][v] = fmaf(c.hk1rc3, dif.x, f[SYY][v]);
    f[SXY][v] = fmaf(c.hk2rc2, dif.y, f[SXY][v]);
  }
}

// x-sweep of one lane's V nodes: FP32 in the difference form (invariant pairs packed when
// XPACK), FP64 in the reference's flux form.
template <typename T, int V, bool XPACK = true>
__device__ __forceinline__ void sweep_x_lane(T (&f)[NF][V], const Sweep<T>& c) {
  if constexpr (sizeof(T) == 8)
    sweep_x_lane_exact<V>(f, c);
  else if constexpr (XPACK)
    sweep_x_lane_packed<V>(f, c);
  else
    sweep_x_lane_diff<T, V>(f, c);
}

// Shared memory of one warp: NPF rows of raw input (filled by cp.async, NPF-1 rows ahead)
// and 3 x-swept rows, each NF fields x 32*V columns.
template <typename T, int V, int NPF>
__host__ __device__ constexpr int warp_smem_elems() {
  return (3 + NPF) * NF * 32 * V;
}

// Asynchronous global -> shared copy of one lane's V columns of one field (L2 only for
// 16-byte pieces, so it is also safe when other warps of the launch wrote the source).
template <int BYTES>
__device__ __forceinline__ void cp_async(void* smem, const void* gmem) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  if (BYTES == 16)
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(s), "l"(gmem) : "memory");
  else
    asm volatile("cp.async.ca.shared.global [%0], [%1], %2;" ::"r"(s), "l"(gmem), "n"(BYTES)
                 : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

// Stores of one lane's V columns that only the lanes with `p` set perform (a predicated
// store, not a branch around it).  Memory clobbers keep them ordered with the fences and
// release stores that publish a tile in the batched kernel.
__device__ __forceinline__ void store_if(bool p, float4* a, const float4& v) {
  asm volatile(
      "{\n\t.reg .pred q;\n\tsetp.ne.u32 q, %0, 0;\n\t@q st.global.v4.f32 [%1], {%2, %3, %4, %5};\n\t}" ::"r"(
          (unsigned)p),
      "l"(a), "f"(v.x), "f"(v.y), "f"(v.z), "f"(v.w)
      : "memory");
}
__device__ __forceinline__ void store_if(bool p, float2* a, const float2& v) {
  asm volatile("{\n\t.reg .pred q;\n\tsetp.ne.u32 q, %0, 0;\n\t@q st.global.v2.f32 [%1], {%2, %3};\n\t}" ::"r"(
                   (unsigned)p),
               "l"(a), "f"(v.x), "f"(v.y)
               : "memory");
}
__device__ __forceinline__ void store_if(bool p, double2* a, const double2& v) {
  asm volatile("{\n\t.reg .pred q;\n\tsetp.ne.u32 q, %0, 0;\n\t@q st.global.v2.f64 [%1], {%2, %3};\n\t}" ::"r"(
                   (unsigned)p),
               "l"(a), "d"(v.x), "d"(v.y)
               : "memory");
}
__device__ __forceinline__ void store_if(bool p, double* a, const double& v) {
  asm volatile("{\n\t.reg .pred q;\n\tsetp.ne.u32 q, %0, 0;\n\t@q st.global.f64 [%1], %2;\n\t}" ::"r"(
                   (unsigned)p),
               "l"(a), "d"(v)
               : "memory");
}

// Element i of a lane's V values (a select chain: i is not a compile-time index).
template <typename T, int V>
__device__ __forceinline__ T pick(const T (&a)[V], int i) {
  T s = a[0];
#pragma unroll
  for (int j = 1; j < V; ++j) s = i == j ? a[j] : s;
  return s;
}

// The first column of the aligned V-column chunk a lane of a strip that reaches past the
// grid edge copies: its own columns clamped into [0, nx) all lie in it, and it lies inside
// the row's pitch (rows are padded to whole chunks).
template <int V>
__device__ __forceinline__ int chunk_col(int col0, int nx) {
  return min(max(col0, 0), (nx - 1) / V * V);
}

// Starts copying source row `row` into this lane's slot of the input ring.  A strip that
// reaches past the grid edge copies each lane's chunk_col() chunk instead; clamp_lane()
// then gives the lane's columns outside [0, nx) the values of column 0 / nx-1.
template <typename T, int V, bool COHERENT>
__device__ __forceinline__ void fetch_row(T* slot, const GridRef<T>& g, int row, int col0,
                                          bool interior) {
  constexpr int kIn = 32 * V;
  const T* base = g.src + (long long)row * g.pitch + (interior ? col0 : chunk_col<V>(col0, g.nx));
#pragma unroll
  for (int k = 0; k < NF; ++k) {
    const T* p = base + k * g.plane;
    if (in_src(g, p, V)) cp_async<V * (int)sizeof(T)>(slot + k * kIn, p);
  }
  cp_async_commit();
}

// The lane's values of a row fetched from its chunk_col() chunk, as the clamped columns
// col0 .. col0+V-1: its own columns where the chunk starts at col0 (positions up to nx-1),
// the chunk's column 0 (left of the grid) or nx-1 (right of it) for the others.
template <typename T, int V>
__device__ __forceinline__ void clamp_lane(T (&f)[NF][V], int col0, int nx) {
  const int c0 = chunk_col<V>(col0, nx);
  const int last = col0 < 0 ? 0 : min(nx - 1 - c0, V - 1);  // position of the edge column
  const int keep = c0 == col0 ? last : -1;                   // own columns: positions [0, keep]
#pragma unroll
  for (int k = 0; k < NF; ++k) {
    const T e = pick<T, V>(f[k], last);
#pragma unroll
    for (int v = 0; v < V; ++v) f[k][v] = v <= keep ? f[k][v] : e;
  }
}

// The per-column y-pipeline.  Row m arrives x-swept; with row m-1 it gives the face
// differences D_{m-1}.  left() advances the left-moving invariants, apply() adds the
// increments of row m-2 to its fields, right() advances the right-moving invariants.
// Face j lies between rows j and j+1.
template <typename T, int V>
struct YPipe;

// FP64: the reference's flux form (as sweep_x_lane_exact, along y).  left() forms
// G_{m-1} = w_{m-1} - psi'_{m-1} D_{m-2} and the left-moving flux difference of row m-2,
// G_{m-2} - G_{m-1}; apply() completes row m-2 from its invariants and both flux
// differences; right() forms F_{m-1} = w_{m-1} + psi_{m-1} D_{m-1} and the right-moving
// flux difference of row m-1, F_{m-1} - F_{m-2}.  State: for w1/w3 P_{m-2}, F_{m-2} and
// that difference; for w2/w4 Q_{m-2}, D_{m-2}, G_{m-2}.
template <int V>
struct YPipe<double, V> {
  double p2[2][V], f2[2][V], dr[2][V], q2[2][V], d2[2][V], g2[2][V];
  double dfw[2][V], wr[2][V], dl[2][V];  // this row's D_{m-1} and w_{m-1} of w1/w3; row m-2's left difference

  __device__ __forceinline__ void init() {
#pragma unroll
    for (int v = 0; v < V; ++v)
#pragma unroll
      for (int q = 0; q < 2; ++q) p2[q][v] = f2[q][v] = dr[q][v] = q2[q][v] = d2[q][v] = g2[q][v] = 0.0;
  }

  __device__ __forceinline__ void left(const double (&f)[NF][V], const double (&pvy)[V],
                                       const double (&psyy)[V], const double (&pvx)[V],
                                       const double (&psxy)[V], const Sweep<double>& cy) {
    const double eps = tvd_eps<double>();
#pragma unroll
    for (int v = 0; v < V; ++v) {
      double wc[4], wp[4];  // invariants of rows m and m-1 (omega_y: vn = vy, sn = syy, vt = vx)
      ex::invariants(f[VY][v], f[SYY][v], f[VX][v], f[SXY][v], cy, wc);
      ex::invariants(pvy[v], psyy[v], pvx[v], psxy[v], cy, wp);
#pragma unroll
      for (int q = 0; q < 2; ++q) {
        const double kc = q ? cy.kc2 : cy.kc1;
        dfw[q][v] = ex::sub(wc[2 * q], wp[2 * q]);
        wr[q][v] = wp[2 * q];
        const double dd = ex::sub(wc[2 * q + 1], wp[2 * q + 1]);
        const double q1 = ex::sub(eps, dd);
        const double ps = psi_ratio(q1, q2[q][v], kc);
        const double g1 = ex::sub(wp[2 * q + 1], ex::mul(ps, d2[q][v]));
        dl[q][v] = ex::sub(g2[q][v], g1);
        g2[q][v] = g1;
        d2[q][v] = dd;
        q2[q][v] = q1;
      }
    }
  }

  __device__ __forceinline__ void apply(double (&gf)[NF][V], const Sweep<double>& cy) const {
#pragma unroll
    for (int v = 0; v < V; ++v) {
      double w[4];
      ex::invariants(gf[VY][v], gf[SYY][v], gf[VX][v], gf[SXY][v], cy, w);
      const double c1 = ex::change(w[0], cy.k1, dr[0][v]);
      const double c2 = ex::change(w[1], cy.k1, dl[0][v]);
      const double c3 = ex::change(w[2], cy.k2, dr[1][v]);
      const double c4 = ex::change(w[3], cy.k2, dl[1][v]);
      ex::increment<1>(gf[VX][v], gf[VY][v], gf[SXX][v], gf[SXY][v], gf[SYY][v], c1, c2, c3, c4, cy);
    }
  }

  __device__ __forceinline__ void right(const Sweep<double>& cy) {
    const double eps = tvd_eps<double>();
#pragma unroll
    for (int v = 0; v < V; ++v) {
#pragma unroll
      for (int q = 0; q < 2; ++q) {
        const double kc = q ? cy.kc2 : cy.kc1;
        const double dd = dfw[q][v];
        const double p1 = ex::add(dd, eps);
        const double ps = psi_ratio(p2[q][v], p1, kc);
        const double f1 = ex::add(wr[q][v], ex::mul(ps, dd));
        dr[q][v] = ex::sub(f1, f2[q][v]);
        f2[q][v] = f1;
        p2[q][v] = p1;
      }
    }
  }
};

// FP32: the same pipeline on pairs of columns with packed f32x2 arithmetic (the columns
// are independent in the y-sweep).  Signs are arranged so that no negation is needed:
// the right-moving state keeps -t and -A.  Reciprocals and the limiter's min/max/sat stay
// per element.

template <int V>
struct YPipe<float, V> {
  static_assert(V % 2 == 0, "pairs of columns");
  static constexpr int P = V / 2;
  float2 p2[2][P], nt2[2][P], na2[2][P], q2[2][P], d2[2][P], c2[2][P];
  float2 dfw[2][P], bo[2][P];

  __device__ __forceinline__ void init() {
#pragma unroll
    for (int i = 0; i < P; ++i)
#pragma unroll
      for (int q = 0; q < 2; ++q) p2[q][i] = nt2[q][i] = na2[q][i] = q2[q][i] = d2[q][i] = c2[q][i] = f2(0.f, 0.f);
  }

  // The constants come as pairs (YPairs); the Sweep overloads pair them up in registers.
  __device__ __forceinline__ void left(const float (&f)[NF][V], const float (&pvy)[V],
                                       const float (&psyy)[V], const float (&pvx)[V],
                                       const float (&psxy)[V], const YPairs& yc) {
    const float2 m1 = f2(-1.f, -1.f), eps = f2(1e-6f, 1e-6f);
#pragma unroll
    for (int i = 0; i < P; ++i) {
      const int a = 2 * i, b = 2 * i + 1;
      const float2 dvn = fma2(f2(pvy[a], pvy[b]), m1, f2(f[VY][a], f[VY][b]));
      const float2 dsn = fma2(f2(psyy[a], psyy[b]), m1, f2(f[SYY][a], f[SYY][b]));
      const float2 dvt = fma2(f2(pvx[a], pvx[b]), m1, f2(f[VX][a], f[VX][b]));
      const float2 dsx = fma2(f2(psxy[a], psxy[b]), m1, f2(f[SXY][a], f[SXY][b]));
      const float2 d[4] = {fma2(dsn, yc.nir1, dvn), fma2(dsn, yc.ir1, dvn), fma2(dsx, yc.nir2, dvt),
                           fma2(dsx, yc.ir2, dvt)};
#pragma unroll
      for (int q = 0; q < 2; ++q) {
        dfw[q][i] = d[2 * q];
        const float2 dd = d[2 * q + 1];
        const float2 q1 = fma2(dd, m1, eps);  // eps - D
        const float2 phi = superbee2(ratio2(q1, q2[q][i]));
        const float2 ps = mul2(q ? yc.k2 : yc.k1, phi), nps = mul2(q ? yc.nk2 : yc.nk1, phi);
        bo[q][i] = fma2(nps, d2[q][i], c2[q][i]);  // c - psi' D_{m-2}
        c2[q][i] = fma2(ps, d2[q][i], dd);         // D + psi' D_{m-2}
        d2[q][i] = dd;
        q2[q][i] = q1;
      }
    }
  }
  __device__ __forceinline__ void left(const float (&f)[NF][V], const float (&pvy)[V],
                                       const float (&psyy)[V], const float (&pvx)[V],
                                       const float (&psxy)[V], const Sweep<float>& cy) {
    left(f, pvy, psyy, pvx, psxy, make_ypairs(cy));
  }

  __device__ __forceinline__ void apply(float (&gf)[NF][V], const YPairs& yc) const {
    const float2 m1 = f2(-1.f, -1.f);
#pragma unroll
    for (int i = 0; i < P; ++i) {
      const int a = 2 * i, b = 2 * i + 1;
      const float2 s1 = fma2(na2[0][i], m1, bo[0][i]);  // A1 + B2
      const float2 p1 = add2(bo[0][i], na2[0][i]);     // B2 - A1
      const float2 s3 = fma2(na2[1][i], m1, bo[1][i]);  // A3 + B4
      const float2 p3 = add2(bo[1][i], na2[1][i]);     // B4 - A3
      const float2 vy = fma2(yc.hk1, s1, f2(gf[VY][a], gf[VY][b]));
      const float2 vx = fma2(yc.hk2, s3, f2(gf[VX][a], gf[VX][b]));
      const float2 syy = fma2(yc.hk1rc1, p1, f2(gf[SYY][a], gf[SYY][b]));
      const float2 sxx = fma2(yc.hk1rc3, p1, f2(gf[SXX][a], gf[SXX][b]));
      const float2 sxy = fma2(yc.hk2rc2, p3, f2(gf[SXY][a], gf[SXY][b]));
      gf[VY][a] = vy.x; gf[VY][b] = vy.y;
      gf[VX][a] = vx.x; gf[VX][b] = vx.y;
      gf[SYY][a] = syy.x; gf[SYY][b] = syy.y;
      gf[SXX][a] = sxx.x; gf[SXX][b] = sxx.y;
      gf[SXY][a] = sxy.x; gf[SXY][b] = sxy.y;
    }
  }
  __device__ __forceinline__ void apply(float (&gf)[NF][V], const Sweep<float>& cy) const {
    apply(gf, make_ypairs(cy));
  }

  __device__ __forceinline__ void right(const YPairs& yc) {
    const float2 eps = f2(1e-6f, 1e-6f);
#pragma unroll
    for (int i = 0; i < P; ++i) {
#pragma unroll
      for (int q = 0; q < 2; ++q) {
        const float2 dd = dfw[q][i];
        const float2 p1 = add2(dd, eps);
        const float2 phi = superbee2(ratio2(p2[q][i], p1));
        const float2 ps = mul2(q ? yc.k2 : yc.k1, phi), nps = mul2(q ? yc.nk2 : yc.nk1, phi);
        na2[q][i] = fma2(ps, dd, nt2[q][i]);  // -(t_{m-2} - psi D)
        nt2[q][i] = fma2(nps, dd, dd);        // -(psi - 1) D
        p2[q][i] = p1;
      }
    }
  }
  __device__ __forceinline__ void right(const Sweep<float>& cy) { right(make_ypairs(cy)); }
};

// Advances one tile -- strip `strip` (32*V columns, halo lanes included), rows [y0, y1) --
// by one step from g.src to g.dst (XPACK: the x-sweep's form, see sweep_x_lane).  `smem_warp` = this warp's warp_smem_elems() elements of
// shared memory; every lane touches only its own V columns of it.  Called by all 32 lanes.
template <typename T, int V, int NPF, bool COHERENT, bool TAP, bool XPACK = true>
__device__ __forceinline__ void march_tile(const GridRef<T>& g, const StepConsts<T>& c, int strip,
                                           int y0, int y1, T* smem_warp, const RowTap<T>& tap) {
  using VT = typename Vec<T, V>::type;
  static_assert(!COHERENT || V * sizeof(T) == 16, "coherent loads need 16-byte (L2-only) copies");
  static_assert(NPF >= 2, "the input ring needs at least the current and the next row");
  constexpr int H = halo_lanes(V);
  constexpr int kIn = 32 * V;
  constexpr int kOut = strip_cols(V);
  constexpr int kRow = NF * kIn;  // elements of one ring slot
  const int lane = threadIdx.x & 31;
  T* in_ring = smem_warp + lane * V;  // NPF slots of raw rows
  T* xs_ring = in_ring + NPF * kRow;  // 3 slots of x-swept rows
  const int xs = strip * kOut - H * V;
  const int col0 = xs + lane * V;
  const bool interior = xs >= 0 && xs + kIn <= g.nx;
  const bool writer = lane >= H && lane < 32 - H && col0 < g.nx;
  const Sweep<T>& cy = c.y;

  // y-pipeline; the fields of row m-1 that enter the y-differences are read back from the
  // x-swept ring
  YPipe<T, V> yp;
  yp.init();
  // the slot read as "row y0-3" by the first row: zero, so no stale shared memory enters
#pragma unroll
  for (int k = 0; k < NF; ++k) *reinterpret_cast<VT*>(xs_ring + 2 * kRow + k * kIn) = VT{};

#pragma unroll
  for (int j = 0; j < NPF - 1; ++j)
    fetch_row<T, V, COHERENT>(in_ring + j * kRow, g, source_row(y0 - 2 + j, g.ny, g.far_rot), col0,
                              interior);
  int islot = 0;  // input slot of row m
  int xslot = 0;  // x-swept slot of row m; row m-1 in (xslot + 2) % 3, row m-2 in (xslot + 1) % 3
  for (int m = y0 - 2; m < y1 + 2; ++m) {
    {
      const int mm = m + NPF - 1;
      const int ns = islot + NPF - 1 >= NPF ? islot - 1 : islot + NPF - 1;
      if (mm < y1 + 2)
        fetch_row<T, V, COHERENT>(in_ring + ns * kRow, g, source_row(mm, g.ny, g.far_rot), col0,
                                  interior);
      else
        cp_async_commit();  // keep one group per row
    }
    cp_async_wait<NPF - 1>();  // row m has landed
    T f[NF][V];
#pragma unroll
    for (int k = 0; k < NF; ++k)
      unpack(*reinterpret_cast<const VT*>(in_ring + islot * kRow + k * kIn), f[k]);
    if (!interior) clamp_lane<T, V>(f, col0, g.nx);

    sweep_x_lane<T, V, XPACK>(f, c.x);

    T* rs = xs_ring + xslot * kRow;
#pragma unroll
    for (int k = 0; k < NF; ++k) *reinterpret_cast<VT*>(rs + k * kIn) = pack(f[k]);
    // rows m and m-1 as the y-pipeline reads them (16-byte loads land in aligned register
    // groups, which the packed FP32 pipeline consumes without moves)
    const T* rp = xs_ring + (xslot == 0 ? 2 : xslot - 1) * kRow;  // row m-1
    T cur[NF][V], pvy[V], psyy[V], pvx[V], psxy[V];
    unpack(*reinterpret_cast<const VT*>(rs + VY * kIn), cur[VY]);
    unpack(*reinterpret_cast<const VT*>(rs + SYY * kIn), cur[SYY]);
    unpack(*reinterpret_cast<const VT*>(rs + VX * kIn), cur[VX]);
    unpack(*reinterpret_cast<const VT*>(rs + SXY * kIn), cur[SXY]);
    unpack(*reinterpret_cast<const VT*>(rp + VY * kIn), pvy);
    unpack(*reinterpret_cast<const VT*>(rp + SYY * kIn), psyy);
    unpack(*reinterpret_cast<const VT*>(rp + VX * kIn), pvx);
    unpack(*reinterpret_cast<const VT*>(rp + SXY * kIn), psxy);

    // D_{m-1} of the four invariants; left-moving part first: B_{m-2}, c_{m-1}
    yp.left(cur, pvy, psyy, pvx, psxy, cy);

    if (m >= y0 + 2) {  // row m-2 is complete (whole warp computes; stores are predicated)
      const int row = m - 2;
      const T* rg = xs_ring + (xslot == 2 ? 0 : xslot + 1) * kRow;
      T gf[NF][V];
#pragma unroll
      for (int k = 0; k < NF; ++k) unpack(*reinterpret_cast<const VT*>(rg + k * kIn), gf[k]);
      yp.apply(gf, cy);
      T* out = g.dst + (long long)row * g.pitch + col0;
#pragma unroll
      for (int k = 0; k < NF; ++k)
        store_if(writer && in_dst(g, out + k * g.plane, V), reinterpret_cast<VT*>(out + k * g.plane), pack(gf[k]));
      if (TAP && row == tap.row && writer && in_line(col0, V, g.pitch)) {
        *reinterpret_cast<VT*>(tap.out + col0) = pack(gf[VX]);
        *reinterpret_cast<VT*>(tap.out + g.pitch + col0) = pack(gf[VY]);
      }
    }

    // right-moving part: psi_{m-1}, A_{m-1} = t_{m-2} - psi_{m-1} D_{m-1}, t_{m-1}
    yp.right(cy);
    islot = islot + 1 == NPF ? 0 : islot + 1;
    xslot = xslot == 2 ? 0 : xslot + 1;
  }
}

}  // namespace march
}  // namespace le2d
