// Launchers of the device kernels (host side).  All take device pointers to the
// SoA state: field k, row j, column i at base[k * plane + j * pitch + i].
#pragma once

#include <cuda_runtime.h>
#include <stddef.h>

#include "le2d_device.cuh"

namespace le2d {

// Work decomposition of the fused step: the grid is cut into vertical strips of
// strip_out columns (one warp each) and each strip into segments of seg_len rows.
struct FusedPlan {
  int nstrips = 0, seg_len = 0, nsegs = 0, ntasks = 0;
  int blocks = 0, threads = 0;
  size_t smem = 0;
};

// Outputs per warp strip: 30 of the 32 lanes, V = 16 / sizeof(T) columns each.
template <typename T>
constexpr int strip_out() { return 30 * (16 / (int)sizeof(T)); }

template <typename T>
FusedPlan plan_fused(int nx, int ny, int resident_warps, int min_seg);

// Warps of the fused kernel that fit on the device at once.
template <typename T>
int fused_resident_warps(int device);

// One fused time step src -> dst.  far_rot selects the le_step_soa far-end rows.
template <typename T>
cudaError_t launch_fused_step(const T* src, T* dst, int nx, int ny, long long pitch,
                              long long plane, const StepConsts<T>& c, int far_rot,
                              const FusedPlan& plan, cudaStream_t s);

// The plain scheme: one sweep (axis 0 = x, 1 = y) src -> dst, one thread per node, the
// reference's tvd2 formula node by node (two divisions per invariant).
template <typename T>
cudaError_t launch_split_sweep(int axis, const T* src, T* dst, int nx, int ny, long long pitch,
                               long long plane, const Sweep<T>& c, T k1, T k2, int far_rot,
                               cudaStream_t s);

// Contiguous host-layout grid (ST_AOS: [j][i][5], ST_SOA: [5][j][i]) <-> pitched SoA.
template <typename T>
cudaError_t launch_pack(const T* raw, T* soa, int nx, int ny, long long pitch, long long plane,
                        int aos, cudaStream_t s);
template <typename T>
cudaError_t launch_unpack(const T* soa, T* raw, int nx, int ny, long long pitch,
                          long long plane, int aos, cudaStream_t s);

// le_set_ball on the device state (same arithmetic as the host loop).
template <typename T>
cudaError_t launch_set_ball(T* soa, int nx, int ny, long long pitch, long long plane, T hx, T hy,
                            T cx, T cy, T r, T s_val, cudaStream_t s);

// FP64 diagnostics: out[0] energy sum (before the h.x*h.y factor), out[1..5] sum of
// squares, out[6..10] max |value| (as ordered bit patterns).  out must be zeroed first.
template <typename T>
cudaError_t launch_diag(const T* soa, int nx, int ny, long long pitch, long long plane,
                        double rho, double a_nn, double a_xy, double a_s, double* out,
                        cudaStream_t s);

}  // namespace le2d
