// Launchers of the device kernels (host side).  All take device pointers to the
// SoA state: field k, row j, column i at base[k * plane + j * pitch + i].
#pragma once

#include <cuda_runtime.h>
#include <stddef.h>

#include "le2d_device.cuh"

namespace le2d {

// Work decomposition of the fused step: the grid is cut into vertical strips of
// strip_out columns (one warp each) and each strip into segments of seg_len rows.
// A strip is 32 lanes x `lanes` columns.  The x-stencil reaches two nodes each way, so
// the outermost halo_lanes() lanes on each side only supply neighbours.
__host__ __device__ constexpr int halo_lanes(int lanes) { return lanes >= 2 ? 1 : 2; }
__host__ __device__ constexpr int strip_cols(int lanes) { return (32 - 2 * halo_lanes(lanes)) * lanes; }
// Two steps per tile: the second step's stencil reaches 4 nodes each way from the strip's
// edge, so ceil(4 / lanes) halo lanes per side.
__host__ __device__ constexpr int halo_lanes2(int lanes) { return (4 + lanes - 1) / lanes; }
__host__ __device__ constexpr int strip_cols2(int lanes) { return (32 - 2 * halo_lanes2(lanes)) * lanes; }

struct FusedPlan {
  int variant = 0, lanes = 0;
  int depth = 1;           // temporal-block depth: steps per launch
  int warps_per_task = 1;  // 2: a producer / consumer warp pair per tile (march_pair.cuh)
  int nstrips = 0, seg_len = 0, nsegs = 0, ntasks = 0;
  int blocks = 0, threads = 0;
  size_t smem = 0;
};

// Compiled kernel variants (columns per lane, register bound, loop unroll).
template <typename T>
int fused_variant_count();
template <typename T>
int fused_variant_lanes(int variant);
template <typename T>
int fused_variant_depth(int variant);

// halves: the task launches in halves (segment length fitted for that schedule).
template <typename T>
FusedPlan plan_fused(int nx, int ny, int variant, int resident_warps, int min_seg, bool halves = false);

// Warps of the fused kernel variant that fit on the device at once.
template <typename T>
int fused_resident_warps(int device, int variant);

// Warp-pair plans: every wait between the warps of a pair is bounded by wait_ns, after
// which the warp sets *status (a device int) and leaves.  stall_task >= 0 is a test hook:
// the producer warp of that tile hands nothing over, so its partner's wait runs out.
struct PairCtl {
  int* status = nullptr;
  unsigned long long wait_ns = 0;
  int stall_task = -1;
};

// One fused launch src -> dst: plan.depth time steps.  far_rot selects the le_step_soa
// far-end rows (depth-1 plans only).
template <typename T>
cudaError_t launch_fused_step(const T* src, T* dst, int nx, int ny, long long pitch,
                              long long plane, const StepConsts<T>& c, int far_rot,
                              const FusedPlan& plan, const PairCtl& pair, cudaStream_t s);

// The same launch writing only some rows: `nranges` (1 or 2) row ranges [lo[r], hi[r]) of
// the ny-row grid, cut into segments of seg_len rows; rows outside them are read (as the
// stencil needs) but not written.
template <typename T>
cudaError_t launch_fused_rows(const T* src, T* dst, int nx, int ny, long long pitch, long long plane,
                              const StepConsts<T>& c, int far_rot, const FusedPlan& plan,
                              const PairCtl& pair, int seg_len, int nranges, const int* lo,
                              const int* hi, cudaStream_t s);

#ifdef LE2D_CHECK
// Bounds-checked build: accesses of the state the step kernels refused (outside the buffer),
// on the current device, since the last call, per translation unit.
unsigned long long check_violations_fused();
unsigned long long check_violations_batch();
#endif

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

// The VTK writer's scalar: |v| of every node as a big-endian float32, rows j outer
// (out: nx*ny words), the same bytes as the host writer computes.
template <typename T>
cudaError_t launch_vtk_speed(const T* soa, int nx, int ny, long long pitch, long long plane,
                             unsigned* out, cudaStream_t s);

// le_set_ball on the device state (same arithmetic as the host loop).
template <typename T>
cudaError_t launch_set_ball(T* soa, int nx, int ny, long long pitch, long long plane, T hx, T hy,
                            T cx, T cy, T r, T s_val, cudaStream_t s);

// ---- batched persistent kernel (batch.cu) ----

// One instance within one launch window (device-resident array).
template <typename T>
struct BatchInst {
  T* buf[2];             // the two state buffers (pitched SoA)
  int nx, ny;
  long long pitch, plane;
  StepConsts<T> c;
  YPairs yq;             // FP32: c.y as pairs for the packed y-pipeline
  int far_rot;           // le_step_soa far-end rows
  int nstrips, nsegs, seg_len;
  int tile_base;         // index of the instance's first tile in the tile list and done[]
  int parity;            // buffer holding the state at window step 0
  int steps;             // steps of this instance in the window
  int depth;             // steps per work item (temporal-block depth); the last item of an
                         // odd step count advances one step
  long long abs_step0;   // steps the instance had done before the window
  T* trace;              // receiver samples [sample][2][pitch], or null
  int trace_row;         // receiver row
  int trace_every;       // steps between samples
  int* fail;             // the instance's failure word (0 = ok); set when a wait of one of
                         // its tiles gives up, after which its work items are skipped
};

struct BatchTile {
  int inst, strip, seg, pad;
};

struct BatchCtl {
  unsigned long long next;  // next work item
  int status;               // 0 = ok, 1 = a wait between the warps of a pair gave up: the
                            // launch ends early and no instance of it has valid results
  int failed;               // instances whose failure word this launch set (a dependency
                            // wait gave up; only those instances are affected)
};

template <typename T>
int batch_lanes();
// Temporal-block depth of the batched kernel for clamped-end (le_step) instances: 2 for
// FP32 (producer / consumer warp pairs), 1 for FP64; le_step_soa instances use 1.
template <typename T>
int batch_depth();
template <typename T>
size_t batch_smem();
template <typename T>
int batch_resident_blocks(int device);
// step_items[r] = work items before window item step r (r = 0..nsteps; an item step
// advances each instance by its depth); done[] and ctl zeroed.
// stall_plus1 > 0 is a test hook: tile (stall_plus1 - 1) never publishes its first step,
// so the waits that depend on it run out and the launch ends with ctl->status = 1.
template <typename T>
cudaError_t launch_batch(const BatchInst<T>* insts, const BatchTile* tiles,
                         const long long* step_items, int nsteps, long long total_items, int* done,
                         BatchCtl* ctl, unsigned long long wait_ns, int stall_plus1,
                         int resident_blocks, cudaStream_t s);

// FP64 diagnostics: out[0] energy sum (before the h.x*h.y factor), out[1..5] sum of
// squares, out[6..10] max |value| (as ordered bit patterns).  out must be zeroed first.
template <typename T>
cudaError_t launch_diag(const T* soa, int nx, int ny, long long pitch, long long plane,
                        double rho, double a_nn, double a_xy, double a_s, double* out,
                        cudaStream_t s);

}  // namespace le2d
