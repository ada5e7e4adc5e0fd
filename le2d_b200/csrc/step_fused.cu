// Fused time step of one solve: x-sweep and y-sweep in one kernel, one read and
// one write of the state per step (le2d simple/le_core.c:605-620: le_step =
// le_step_x then le_step_y, both with Jacobi semantics and clamped ends).
//
// The grid is cut into vertical strips (32 lanes x V columns, one warp each, the
// outer lanes supplying the x-halo) and each strip into segments of seg_len rows;
// every warp marches one strip segment (march.cuh).  Warps are independent, so a
// block is just kWarps of them sharing the launch.  Variants of temporal-block depth 2
// advance each tile by two steps per launch, on one warp (march2.cuh) or on a producer /
// consumer warp pair (march_pair.cuh).
#include <cmath>
#include <type_traits>

#include "march_pair.cuh"

namespace le2d {

namespace {

template <typename T>
struct FusedParams {
  march::GridRef<T> g;
  int nstrips, seg_len, ntasks;
  StepConsts<T> c;
  YPairs yq;     // FP32: c.y as pairs for the packed y-pipeline
  PairCtl pair;  // warp-pair waits
  // interior tiles: strips [s_lo, s_hi) x segments [g_lo, g_hi) (empty when lo >= hi)
  int s_lo, s_hi, g_lo, g_hi;
  // rows the launch writes: segments [0, nseg0) cover rows [lo0, hi0), the rest [lo1, hi1)
  int lo0, hi0, lo1, hi1, nseg0;
};

// Rows [y0, y1) of segment `seg` of the launch's row ranges.
template <typename T>
__device__ __forceinline__ void segment_rows(const FusedParams<T>& p, int seg, int& y0, int& y1) {
  if (seg < p.nseg0) {
    y0 = p.lo0 + seg * p.seg_len;
    y1 = min(y0 + p.seg_len, p.hi0);
  } else {
    y0 = p.lo1 + (seg - p.nseg0) * p.seg_len;
    y1 = min(y0 + p.seg_len, p.hi1);
  }
}

// Tile of a task when the boundary tiles -- the segments above g_lo and from g_hi on, and
// the strips outside [s_lo, s_hi) of the segments between -- come first and the interior
// tiles (in segment-major order) after them.  The boundary tiles take the general loops,
// which are slower per tile than the lean ones: dealt out first, they finish while interior
// tiles still fill the device, and the launch ends on lean tiles.  Measured with the interior
// tiles first instead (the tail of every launch then being boundary tiles on a thinning
// device): 3-9 % slower (8192^2: 177.0 against 181.7 Gnu/s; 4096^2: 146.0 against 155.0;
// 2048 x 8192: 142.0 against 154.3).
template <typename T>
__device__ __forceinline__ void boundary_first(const FusedParams<T>& p, int task, int& strip, int& seg) {
  const int ni = p.s_hi - p.s_lo, ng = p.g_hi - p.g_lo;
  const int nb = p.ntasks - ni * ng;  // boundary tiles
  task = task < nb ? ni * ng + task : task - nb;
  if (task < ni * ng) {
    seg = p.g_lo + task / ni;
    strip = p.s_lo + task % ni;
    return;
  }
  int k = task - ni * ng;
  const int top = p.g_lo * p.nstrips;
  if (k < top) {
    seg = k / p.nstrips;
    strip = k % p.nstrips;
    return;
  }
  k -= top;
  const int side = p.nstrips - ni;  // boundary strips of a middle segment
  if (k < ng * side) {
    seg = p.g_lo + k / side;
    const int j = k % side;
    strip = j < p.s_lo ? j : p.s_hi + (j - p.s_lo);
    return;
  }
  k -= ng * side;
  seg = p.g_hi + k / p.nstrips;
  strip = k % p.nstrips;
}

// The y-sweep constants the interior loops hand to the y-pipeline: pairs for FP32.
__device__ __forceinline__ const YPairs& ycons(const FusedParams<float>& p) { return p.yq; }
__device__ __forceinline__ const Sweep<double>& ycons(const FusedParams<double>& p) { return p.c.y; }

constexpr int kWarps = 4;  // warps per block

template <typename T, int V, int NPF, int D>
__host__ __device__ constexpr int warp_elems() {
  return D == 2 ? march::warp_smem_elems2<T, V, NPF>() : march::warp_smem_elems<T, V, NPF>();
}

template <typename T, int V, int MINB, int NPF, int D, int F>
__global__ void __launch_bounds__(kWarps * 32, MINB) fused_step_kernel(const FusedParams<T> p) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int wib = threadIdx.x >> 5;
  const int task = blockIdx.x * kWarps + wib;
  if (task >= p.ntasks) return;  // whole warp leaves together
  T* smem = reinterpret_cast<T*>(smem_raw) + wib * warp_elems<T, V, NPF, D>();
  int strip = task % p.nstrips;
  int seg = task / p.nstrips;
  if constexpr (F == 2) boundary_first(p, task, strip, seg);
  int y0, y1;
  segment_rows(p, seg, y0, y1);
  if constexpr (D == 1 && F >= 1) {  // interior tiles on the lean loop
    const int xs = strip * strip_cols(V) - halo_lanes(V) * V;
    if (march::tile_is_interior1<T, V>(p.g, xs, y0, y1)) {
      march::march_tile_interior<T, V, NPF>(p.g, p.c, xs, y0, y1, smem);
      return;
    }
  }
  if constexpr (D == 2)
    march::march_tile2<T, V, NPF, false>(p.g, p.c, strip, y0, y1, smem);
  else
    march::march_tile<T, V, NPF, false, false>(p.g, p.c, strip, y0, y1, smem,
                                                march::RowTap<T>{nullptr, -1});
}

// Two-step tiles on warp pairs: W / 2 pairs per block, each with its own shared
// memory and queue barriers.  The barriers are initialised before the block's barrier, so
// both warps of a pair see them, and the pair leaves together (same tile).
template <typename T, int V, int MINB, int NPF, int W, int F>
__global__ void __launch_bounds__(W * 32, MINB) fused_pair_kernel(const FusedParams<T> p) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  constexpr int kPairs = W / 2;
  const int wib = threadIdx.x >> 5;
  const int pair = kPairs == 1 ? 0 : wib >> 1;
  unsigned char* base = smem_raw + pair * march::pair_smem_bytes<T, V, NPF>();
  unsigned long long* bars =
      reinterpret_cast<unsigned long long*>(base + march::pair_smem_elems<T, V, NPF>() * sizeof(T));
  const bool producer = (wib & 1) == 0;
  if (producer) march::pair_init<T, V>(bars);
  __syncthreads();
  const int task = blockIdx.x * kPairs + pair;
  if (task >= p.ntasks) return;  // both warps of the pair
  if (task == p.pair.stall_task && producer) return;  // test hook
  int strip = task % p.nstrips;
  int seg = task / p.nstrips;
  if constexpr (F == 2) boundary_first(p, task, strip, seg);
  int y0, y1;
  segment_rows(p, seg, y0, y1);
  T* smem = reinterpret_cast<T*>(base);
  unsigned u = 0;
  const march::RowTap<T> no_tap{nullptr, -1};
  if constexpr (F >= 1) {  // interior tiles on the lean loops
    const int xs = strip * strip_cols2(V) - halo_lanes2(V) * V;
    if (march::tile_is_interior<T, V>(p.g, xs, y0, y1)) {
      if (producer)
        march::pair_produce_interior<T, V, NPF>(p.g, p.c.x, ycons(p), xs, y0, y1, smem, bars,
                                                p.pair.wait_ns, p.pair.status, u);
      else
        march::pair_consume_interior<T, V, NPF>(p.g, p.c.x, ycons(p), xs, y0, y1, smem, bars,
                                                p.pair.wait_ns, p.pair.status, u);
      return;
    }
  }
  if (producer)
    march::pair_produce<T, V, NPF, false>(p.g, p.c.x, ycons(p), strip, y0, y1, smem, bars, p.pair.wait_ns,
                                          p.pair.status, u, false);
  else
    march::pair_consume<T, V, NPF, false>(p.g, p.c.x, ycons(p), strip, y0, y1, smem, bars, p.pair.wait_ns,
                                          p.pair.status, u, false, no_tap, no_tap);
}

// Compiled variants: columns per lane V (one 16- or 8-byte access per field), the
// minimum resident blocks per SM handed to the register allocator, the depth of the
// shared-memory input ring (NPF - 1 rows are in flight ahead of the row being swept),
// the temporal-block depth D (steps per launch), P = 1 for two-step tiles on warp pairs,
// warps per block W, and F: 1 = interior tiles on the lean loops, 2 = the same with the
// boundary tiles dealt out first (boundary_first: the general loops they take run beside
// the lean ones on an SM only at the start of the launch, which ends on lean tiles).
template <typename T, int VAR>
struct VariantCfg;
template <> struct VariantCfg<float, 0> { static constexpr int V = 4, MINB = 3, NPF = 2, D = 1, P = 0, W = 4, F = 0; };
template <> struct VariantCfg<float, 1> { static constexpr int V = 4, MINB = 3, NPF = 3, D = 1, P = 0, W = 4, F = 0; };
template <> struct VariantCfg<float, 2> { static constexpr int V = 4, MINB = 4, NPF = 2, D = 1, P = 0, W = 4, F = 0; };
template <> struct VariantCfg<float, 3> { static constexpr int V = 2, MINB = 4, NPF = 2, D = 1, P = 0, W = 4, F = 0; };
template <> struct VariantCfg<float, 4> { static constexpr int V = 2, MINB = 4, NPF = 3, D = 1, P = 0, W = 4, F = 0; };
template <> struct VariantCfg<float, 5> { static constexpr int V = 4, MINB = 2, NPF = 2, D = 2, P = 0, W = 4, F = 0; };
template <> struct VariantCfg<float, 6> { static constexpr int V = 2, MINB = 4, NPF = 2, D = 2, P = 0, W = 4, F = 0; };
template <> struct VariantCfg<float, 7> { static constexpr int V = 2, MINB = 3, NPF = 3, D = 2, P = 0, W = 4, F = 0; };
template <> struct VariantCfg<float, 8> { static constexpr int V = 2, MINB = 5, NPF = 2, D = 2, P = 0, W = 4, F = 0; };
template <> struct VariantCfg<float, 9> { static constexpr int V = 4, MINB = 4, NPF = 2, D = 2, P = 1, W = 4, F = 0; };
template <> struct VariantCfg<float, 10> { static constexpr int V = 4, MINB = 3, NPF = 3, D = 2, P = 1, W = 4, F = 0; };
template <> struct VariantCfg<float, 11> { static constexpr int V = 4, MINB = 4, NPF = 2, D = 2, P = 1, W = 4, F = 1; };
template <> struct VariantCfg<float, 12> { static constexpr int V = 4, MINB = 8, NPF = 2, D = 2, P = 1, W = 2, F = 1; };
template <> struct VariantCfg<float, 13> { static constexpr int V = 4, MINB = 8, NPF = 2, D = 2, P = 1, W = 2, F = 2; };
template <> struct VariantCfg<float, 14> { static constexpr int V = 4, MINB = 4, NPF = 2, D = 1, P = 0, W = 4, F = 2; };
template <> struct VariantCfg<float, 15> { static constexpr int V = 4, MINB = 5, NPF = 2, D = 1, P = 0, W = 4, F = 2; };
template <> struct VariantCfg<double, 0> { static constexpr int V = 2, MINB = 2, NPF = 2, D = 1, P = 0, W = 4, F = 0; };
template <> struct VariantCfg<double, 1> { static constexpr int V = 2, MINB = 3, NPF = 2, D = 1, P = 0, W = 4, F = 0; };
template <> struct VariantCfg<double, 2> { static constexpr int V = 1, MINB = 4, NPF = 2, D = 1, P = 0, W = 4, F = 0; };
template <> struct VariantCfg<double, 3> { static constexpr int V = 1, MINB = 4, NPF = 3, D = 1, P = 0, W = 4, F = 0; };
template <> struct VariantCfg<double, 4> { static constexpr int V = 1, MINB = 5, NPF = 2, D = 1, P = 0, W = 4, F = 0; };
template <> struct VariantCfg<double, 5> { static constexpr int V = 2, MINB = 2, NPF = 2, D = 2, P = 0, W = 4, F = 0; };
template <> struct VariantCfg<double, 6> { static constexpr int V = 1, MINB = 4, NPF = 2, D = 2, P = 0, W = 4, F = 0; };
template <> struct VariantCfg<double, 7> { static constexpr int V = 1, MINB = 3, NPF = 3, D = 2, P = 0, W = 4, F = 0; };
template <> struct VariantCfg<double, 8> { static constexpr int V = 1, MINB = 5, NPF = 2, D = 2, P = 0, W = 4, F = 0; };
template <> struct VariantCfg<double, 9> { static constexpr int V = 2, MINB = 3, NPF = 2, D = 2, P = 1, W = 4, F = 0; };
template <> struct VariantCfg<double, 10> { static constexpr int V = 2, MINB = 4, NPF = 2, D = 2, P = 1, W = 4, F = 0; };
template <> struct VariantCfg<double, 11> { static constexpr int V = 2, MINB = 3, NPF = 2, D = 2, P = 1, W = 4, F = 1; };
template <> struct VariantCfg<double, 12> { static constexpr int V = 2, MINB = 6, NPF = 2, D = 2, P = 1, W = 2, F = 1; };
template <> struct VariantCfg<double, 13> { static constexpr int V = 2, MINB = 6, NPF = 2, D = 2, P = 1, W = 2, F = 2; };
template <> struct VariantCfg<double, 14> { static constexpr int V = 2, MINB = 2, NPF = 2, D = 1, P = 0, W = 4, F = 2; };
template <> struct VariantCfg<double, 15> { static constexpr int V = 2, MINB = 4, NPF = 2, D = 1, P = 0, W = 4, F = 2; };
constexpr int kVariants = 16;

template <typename T, int VAR>
struct VariantKernel {
  using C = VariantCfg<T, VAR>;
  static_assert(C::P == 1 || C::W == kWarps, "block size: warp pairs only");
  static_assert(C::P == 1 || C::D == 1 || C::F == 0, "lean loops: warp pairs and one-step tiles");
  static void* fn() {
    if constexpr (C::P == 1)
      return (void*)fused_pair_kernel<T, C::V, C::MINB, C::NPF, C::W, C::F>;
    else
      return (void*)fused_step_kernel<T, C::V, C::MINB, C::NPF, C::D, C::F>;
  }
  static size_t smem() {
    if constexpr (C::P == 1)
      return (size_t)(C::W / 2) * march::pair_smem_bytes<T, C::V, C::NPF>();
    else
      return (size_t)kWarps * warp_elems<T, C::V, C::NPF, C::D>() * sizeof(T);
  }
  // dynamic shared memory above 48 KB must be opted into once per kernel and device
  static void prepare() {
    static unsigned long long done = 0;  // bit d: device d (devices 0..63)
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) {
      cudaFuncSetAttribute(fn(), cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem());
      return;
    }
    if (!(done & (1ull << dev))) {
      cudaFuncSetAttribute(fn(), cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem());
      done |= 1ull << dev;
    }
  }
  static void launch(const FusedPlan& pl, const FusedParams<T>& p, cudaStream_t s) {
    if constexpr (C::P == 1)
      fused_pair_kernel<T, C::V, C::MINB, C::NPF, C::W, C::F><<<pl.blocks, pl.threads, pl.smem, s>>>(p);
    else
      fused_step_kernel<T, C::V, C::MINB, C::NPF, C::D, C::F><<<pl.blocks, pl.threads, pl.smem, s>>>(p);
  }
};

template <typename T, template <typename, int> class Op, typename R, typename... A>
R with_variant(int var, A&&... a) {
  switch (var) {
    case 1: return Op<T, 1>::run(a...);
    case 2: return Op<T, 2>::run(a...);
    case 3: return Op<T, 3>::run(a...);
    case 4: return Op<T, 4>::run(a...);
    case 5: return Op<T, 5>::run(a...);
    case 6: return Op<T, 6>::run(a...);
    case 7: return Op<T, 7>::run(a...);
    case 8: return Op<T, 8>::run(a...);
    case 9: return Op<T, 9>::run(a...);
    case 10: return Op<T, 10>::run(a...);
    case 11: return Op<T, 11>::run(a...);
    case 12: return Op<T, 12>::run(a...);
    case 13: return Op<T, 13>::run(a...);
    case 14: return Op<T, 14>::run(a...);
    case 15: return Op<T, 15>::run(a...);
    default: return Op<T, 0>::run(a...);
  }
}

template <typename T, int VAR>
struct LanesOp {
  static int run() { return VariantCfg<T, VAR>::V; }
};
template <typename T, int VAR>
struct DepthOp {
  static int run() { return VariantCfg<T, VAR>::D; }
};
template <typename T, int VAR>
struct PairOp {
  static int run() { return VariantCfg<T, VAR>::P; }
};
template <typename T, int VAR>
struct WarpsOp {
  static int run() { return VariantCfg<T, VAR>::W; }
};
template <typename T, int VAR>
struct ResidentOp {
  static int run(int device) {
    int sms = 0, per_sm = 0;
    VariantKernel<T, VAR>::prepare();
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device) != cudaSuccess) return 0;
    constexpr int W = VariantCfg<T, VAR>::W;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, VariantKernel<T, VAR>::fn(), W * 32,
                                                      VariantKernel<T, VAR>::smem()) != cudaSuccess)
      return 0;
    return sms * per_sm * W;
  }
};
template <typename T, int VAR>
struct SmemOp {
  static size_t run() {
    VariantKernel<T, VAR>::prepare();
    return VariantKernel<T, VAR>::smem();
  }
};
template <typename T, int VAR>
struct LaunchOp {
  static int run(const FusedPlan& pl, const FusedParams<T>& p, cudaStream_t s) {
    VariantKernel<T, VAR>::prepare();  // the launching device may not have planned it
    VariantKernel<T, VAR>::launch(pl, p, s);
    return 0;
  }
};

}  // namespace

template <typename T>
int fused_variant_count() { return kVariants; }

template <typename T>
int fused_variant_lanes(int variant) { return with_variant<T, LanesOp, int>(variant); }

template <typename T>
int fused_variant_depth(int variant) { return with_variant<T, DepthOp, int>(variant); }

template <typename T>
int fused_resident_warps(int device, int variant) {
  return with_variant<T, ResidentOp, int>(variant, device);
}

// Segments are sized so the launch runs several waves of warps (kWaves): blocks are
// dispatched in task order, so the warps resident at any moment cover one band of
// neighbouring rows -- DRAM pages shared by adjacent strips, halo rows shared in L2 --
// rather than rows a long segment apart.  Measured on the 8192^2 FP32 case: 32-row
// segments (8 waves) run at 1.33e11 node-updates/s, single-wave 241-row segments at 1.0e11.
// A two-step tile recomputes 8 halo rows of step A and 4 of step B, so its segments are
// at least twice min_seg (at 4096^2: 32-row segments 1.17e11, 16-row 1.09e11).
constexpr int kWaves = 8;

// The segment length L that minimises a model of the launch time fitted to measured
// launches,
//   time ~ (w + beta + alpha (ceil(w) - w)) (L + h) (1 + kappa L / 128),   w = tiles / resident tiles,
// w being the launch's waves of tiles, L + h the rows of a tile's march (h for its halo rows
// and the fill of its pipeline), alpha the charge for the idle part of the last wave and
// kappa one for long tiles (the tiles resident at a time then span more rows of the grid).
// L is one of the lengths the fit measured.  Fits:
//   warp-pair (two-step) variants, the FP32 default with its boundary tiles dealt out first,
//   measured on 2048^2 to 16384^2, 8192 x 2048 and 2048 x 8192 with segments of 32 to 256
//   rows: h = 10, beta = 0.1, alpha = 0.5, kappa = 0.02 -- the fastest measured length on
//   each of those grids (an earlier fit without the length term: up to 7 % below it, e.g.
//   147.4 against 158.3 Gnu/s on 3000^2, 155.1 against 158.4 on 4096^2; the earlier rule of
//   about 8 waves of tiles: up to 13 % below it);
//   warp-pair variants launched in halves (le2d_api.cu), w counting the tiles of one half:
//   h = 14, beta = 0, alpha = 0.2, kappa = 0 -- fitted on the same grids with the halves
//   forced on, it picks the fastest measured length, and the halves with it beat the best
//   whole launches on each of those grids but 2048^2 (2 % below): e.g. 4096^2 176.2 against
//   158.5, 8192 x 2048 179.5 against 158.7, 8192^2 195.2 against 181.8 Gnu/s;
//   FP64 one-step variants, the FP64 default measured on 2048^2 to 12000^2 and 8192 x 2048
//   with segments of 16 to 128 rows: h = 8, beta = 0.3, alpha = 0, kappa = 0.1 -- within 1 %
//   of the fastest measured length on each (the 8-wave rule: up to 10 % below it, e.g. 40.3
//   against 44.2 Gnu/s on 2048^2, 46.6 against 51.3 on 4096^2); launched in halves, with the
//   waves of one half, h = 8, beta = 0, alpha = 0.2, kappa = 0.1 -- the fastest measured length
//   on each (2-3 % above the whole launches' lengths in halves: 8192^2 58.8 against 57.3,
//   2048^2 48.1 against 46.5 Gnu/s).
struct SegModel {
  double h, beta, alpha, kappa;
  const int* lens;
  int nlens;
};
constexpr int kPairLens[] = {32, 48, 64, 80, 96, 128, 160, 192, 256};
constexpr int kStepLensF64[] = {16, 24, 32, 40, 48, 56, 64, 80, 96, 112, 128};
constexpr SegModel kPairModel{10.0, 0.1, 0.5, 0.02, kPairLens, 9};
constexpr SegModel kPairHalvesModel{14.0, 0.0, 0.2, 0.0, kPairLens, 9};
constexpr SegModel kStepModelF64{8.0, 0.3, 0.0, 0.1, kStepLensF64, 11};
constexpr int kStepHalvesLensF64[] = {16, 24, 32, 48, 64, 96, 128};
constexpr SegModel kStepHalvesModelF64{8.0, 0.0, 0.2, 0.1, kStepHalvesLensF64, 7};

inline int model_segment(const SegModel& m, int ny, int nstrips, int resident_tiles, int min_len) {
  int best_len = min_len < ny ? min_len : ny;
  double best = 1e300;
  for (int i = 0; i < m.nlens; ++i) {
    if (m.lens[i] < min_len) continue;
    const int l = m.lens[i] < ny ? m.lens[i] : ny;
    const double w = (double)nstrips * ((ny + l - 1) / l) / resident_tiles;
    const double t = (w + m.beta + m.alpha * (std::ceil(w) - w)) * (l + m.h) * (1.0 + m.kappa * l / 128.0);
    if (t < best) {
      best = t;
      best_len = l;
    }
    if (l == ny) break;
  }
  return best_len;
}

template <typename T>
FusedPlan plan_fused(int nx, int ny, int variant, int resident_warps, int min_seg, bool halves) {
  FusedPlan pl;
  pl.variant = variant < 0 || variant >= kVariants ? 0 : variant;
  pl.lanes = fused_variant_lanes<T>(pl.variant);
  pl.depth = fused_variant_depth<T>(pl.variant);
  pl.warps_per_task = with_variant<T, PairOp, int>(pl.variant) ? 2 : 1;
  const int out = pl.depth == 2 ? strip_cols2(pl.lanes) : strip_cols(pl.lanes);
  pl.nstrips = (nx + out - 1) / out;
  const int resident_tasks = resident_warps / pl.warps_per_task;
  int target = resident_tasks > 0 ? kWaves * resident_tasks / pl.nstrips : 1;
  if (target < 1) target = 1;
  int seg = (ny + target - 1) / target;
  if (seg < min_seg * pl.depth) seg = min_seg * pl.depth;
  if (resident_tasks > 0 && pl.warps_per_task == 2 && halves)  // each half's waves
    seg = model_segment(kPairHalvesModel, ny, pl.nstrips, 2 * resident_tasks, min_seg * pl.depth);
  else if (resident_tasks > 0 && pl.warps_per_task == 2)
    seg = model_segment(kPairModel, ny, pl.nstrips, resident_tasks, min_seg * pl.depth);
  else if (resident_tasks > 0 && sizeof(T) == 8 && pl.depth == 1 && halves)
    seg = model_segment(kStepHalvesModelF64, ny, pl.nstrips, 2 * resident_tasks, min_seg);
  else if (resident_tasks > 0 && sizeof(T) == 8 && pl.depth == 1)
    seg = model_segment(kStepModelF64, ny, pl.nstrips, resident_tasks, min_seg);
  if (seg > ny) seg = ny;
  pl.seg_len = seg;
  pl.nsegs = (ny + seg - 1) / seg;
  pl.ntasks = pl.nstrips * pl.nsegs;
  const int warps = with_variant<T, WarpsOp, int>(pl.variant);
  pl.threads = warps * 32;
  const int tasks_per_block = warps / pl.warps_per_task;
  pl.blocks = (pl.ntasks + tasks_per_block - 1) / tasks_per_block;
  pl.smem = with_variant<T, SmemOp, size_t>(pl.variant);
  return pl;
}

template <typename T>
cudaError_t launch_fused_rows(const T* src, T* dst, int nx, int ny, long long pitch, long long plane,
                              const StepConsts<T>& c, int far_rot, const FusedPlan& plan,
                              const PairCtl& pair, int seg_len, int nranges, const int* lo,
                              const int* hi, cudaStream_t s) {
  if (plan.depth == 2 && far_rot) return cudaErrorInvalidValue;  // two steps assume clamped ends
  if (plan.warps_per_task == 2 && pair.status == nullptr) return cudaErrorInvalidValue;
  if (nranges < 1 || nranges > 2 || seg_len < 1) return cudaErrorInvalidValue;
  FusedParams<T> p;
  p.pair = pair;
  p.g = march::GridRef<T>{src, dst, nx, ny, pitch, plane, far_rot};
  p.nstrips = plan.nstrips;
  p.seg_len = seg_len;
  p.lo0 = lo[0];
  p.hi0 = hi[0];
  p.lo1 = nranges == 2 ? lo[1] : 0;
  p.hi1 = nranges == 2 ? hi[1] : 0;
  for (int r = 0; r < nranges; ++r)
    if (lo[r] < 0 || hi[r] > ny || lo[r] > hi[r]) return cudaErrorInvalidValue;
  p.nseg0 = (p.hi0 - p.lo0 + seg_len - 1) / seg_len;
  const int nseg1 = (p.hi1 - p.lo1 + seg_len - 1) / seg_len;
  p.ntasks = plan.nstrips * (p.nseg0 + nseg1);
  if (p.ntasks == 0) return cudaSuccess;
  p.c = c;
  p.yq = YPairs{};
  if constexpr (std::is_same<T, float>::value) p.yq = make_ypairs(c.y);
  {  // the interior tiles' rectangle, dealt out first (tile_is_interior / tile_is_interior1:
     // the strip inside [0, nx), the rows read, 2 per step beyond the tile's, inside [0, ny));
     // an ordering only -- every tile tests itself -- and empty for two ranges
    const int V = plan.lanes, L = seg_len, margin = 2 * plan.depth;
    const int H = (plan.depth == 2 ? halo_lanes2(V) : halo_lanes(V)) * V;
    const int out = plan.depth == 2 ? strip_cols2(V) : strip_cols(V);
    p.s_lo = (H + out - 1) / out;
    p.s_hi = nx - 32 * V + H >= 0 ? (nx - 32 * V + H) / out + 1 : 0;
    if (p.s_hi > plan.nstrips) p.s_hi = plan.nstrips;
    const int base = p.lo0;
    p.g_lo = margin > base ? (margin - base + L - 1) / L : 0;
    p.g_hi = ny - margin - base >= 0 ? (ny - margin - base) / L : 0;
    if (p.g_hi > p.nseg0) p.g_hi = p.nseg0;
    if (p.s_hi < p.s_lo || nranges == 2) p.s_hi = p.s_lo;
    if (p.g_hi < p.g_lo || nranges == 2) p.g_hi = p.g_lo;
  }
  FusedPlan pl = plan;
  pl.ntasks = p.ntasks;
  const int tasks_per_block = plan.threads / 32 / plan.warps_per_task;
  pl.blocks = (p.ntasks + tasks_per_block - 1) / tasks_per_block;
  with_variant<T, LaunchOp, int>(plan.variant, pl, p, s);
  return cudaGetLastError();
}

template <typename T>
cudaError_t launch_fused_step(const T* src, T* dst, int nx, int ny, long long pitch,
                              long long plane, const StepConsts<T>& c, int far_rot,
                              const FusedPlan& plan, const PairCtl& pair, cudaStream_t s) {
  const int lo = 0, hi = ny;
  return launch_fused_rows<T>(src, dst, nx, ny, pitch, plane, c, far_rot, plan, pair, plan.seg_len, 1,
                              &lo, &hi, s);
}

#ifdef LE2D_CHECK
unsigned long long check_violations_fused() {
  unsigned long long v = 0, zero = 0;
  if (cudaMemcpyFromSymbol(&v, march::g_check_violations, sizeof(v)) != cudaSuccess ||
      cudaMemcpyToSymbol(march::g_check_violations, &zero, sizeof(zero)) != cudaSuccess) {
    cudaGetLastError();
    return ~0ULL;  // unreadable: reported as violations
  }
  return v;
}
#endif

#define LE2D_INST(T)                                                                            \
  template int fused_variant_count<T>();                                                        \
  template int fused_variant_lanes<T>(int);                                                     \
  template int fused_variant_depth<T>(int);                                                     \
  template int fused_resident_warps<T>(int, int);                                               \
  template FusedPlan plan_fused<T>(int, int, int, int, int, bool);                              \
  template cudaError_t launch_fused_step<T>(const T*, T*, int, int, long long, long long,       \
                                            const StepConsts<T>&, int, const FusedPlan&,        \
                                            const PairCtl&, cudaStream_t);                      \
  template cudaError_t launch_fused_rows<T>(const T*, T*, int, int, long long, long long,       \
                                            const StepConsts<T>&, int, const FusedPlan&,        \
                                            const PairCtl&, int, int, const int*, const int*,   \
                                            cudaStream_t);
LE2D_INST(float)
LE2D_INST(double)
#undef LE2D_INST

}  // namespace le2d
