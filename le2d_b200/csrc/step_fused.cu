// Fused time step of one solve: x-sweep and y-sweep in one kernel, one read and
// one write of the state per step (le2d simple/le_core.c:605-620: le_step =
// le_step_x then le_step_y, both with Jacobi semantics and clamped ends).
//
// The grid is cut into vertical strips (32 lanes x V columns, one warp each, the
// outer lanes supplying the x-halo) and each strip into segments of seg_len rows;
// every warp marches one strip segment (march.cuh).  Warps are independent, so a
// block is just kWarps of them sharing the launch.
#include "march.cuh"

namespace le2d {

namespace {

template <typename T>
struct FusedParams {
  march::GridRef<T> g;
  int nstrips, seg_len, ntasks;
  StepConsts<T> c;
};

constexpr int kWarps = 4;  // warps per block

template <typename T, int V, int MINB, int UNROLL>
__global__ void __launch_bounds__(kWarps * 32, MINB) fused_step_kernel(const FusedParams<T> p) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int wib = threadIdx.x >> 5;
  const int task = blockIdx.x * kWarps + wib;
  if (task >= p.ntasks) return;  // whole warp leaves together
  T* ring = reinterpret_cast<T*>(smem_raw) + wib * (3 * NF * 32 * V);
  const int strip = task % p.nstrips;
  const int seg = task / p.nstrips;
  const int y0 = seg * p.seg_len;
  const int y1 = min(y0 + p.seg_len, p.g.ny);
  march::march_tile<T, V, UNROLL, false, false>(p.g, p.c, strip, y0, y1, ring,
                                                 march::RowTap<T>{nullptr, -1});
}

// Compiled variants: columns per lane V (one 16- or 8-byte access per field), the
// minimum resident blocks per SM handed to the register allocator, and the unroll of
// the row loop (2 lets the loop-carried y-pipeline state alternate registers).
template <typename T, int VAR>
struct VariantCfg;
template <> struct VariantCfg<float, 0> { static constexpr int V = 4, MINB = 3, UNROLL = 1; };
template <> struct VariantCfg<float, 1> { static constexpr int V = 4, MINB = 1, UNROLL = 2; };
template <> struct VariantCfg<float, 2> { static constexpr int V = 2, MINB = 4, UNROLL = 1; };
template <> struct VariantCfg<float, 3> { static constexpr int V = 2, MINB = 4, UNROLL = 2; };
template <> struct VariantCfg<float, 4> { static constexpr int V = 4, MINB = 3, UNROLL = 2; };
template <> struct VariantCfg<double, 0> { static constexpr int V = 2, MINB = 2, UNROLL = 1; };
template <> struct VariantCfg<double, 1> { static constexpr int V = 2, MINB = 3, UNROLL = 1; };
template <> struct VariantCfg<double, 2> { static constexpr int V = 1, MINB = 4, UNROLL = 1; };
template <> struct VariantCfg<double, 3> { static constexpr int V = 1, MINB = 4, UNROLL = 2; };
template <> struct VariantCfg<double, 4> { static constexpr int V = 1, MINB = 3, UNROLL = 2; };
constexpr int kVariants = 5;

template <typename T, int VAR>
struct VariantKernel {
  using C = VariantCfg<T, VAR>;
  static void* fn() { return (void*)fused_step_kernel<T, C::V, C::MINB, C::UNROLL>; }
  static size_t smem() { return (size_t)kWarps * 3 * NF * 32 * C::V * sizeof(T); }
  static void launch(const FusedPlan& pl, const FusedParams<T>& p, cudaStream_t s) {
    fused_step_kernel<T, C::V, C::MINB, C::UNROLL><<<pl.blocks, pl.threads, pl.smem, s>>>(p);
  }
};

template <typename T, template <typename, int> class Op, typename R, typename... A>
R with_variant(int var, A&&... a) {
  switch (var) {
    case 1: return Op<T, 1>::run(a...);
    case 2: return Op<T, 2>::run(a...);
    case 3: return Op<T, 3>::run(a...);
    case 4: return Op<T, 4>::run(a...);
    default: return Op<T, 0>::run(a...);
  }
}

template <typename T, int VAR>
struct LanesOp {
  static int run() { return VariantCfg<T, VAR>::V; }
};
template <typename T, int VAR>
struct ResidentOp {
  static int run(int device) {
    int sms = 0, per_sm = 0;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device) != cudaSuccess) return 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, VariantKernel<T, VAR>::fn(), kWarps * 32,
                                                      VariantKernel<T, VAR>::smem()) != cudaSuccess)
      return 0;
    return sms * per_sm * kWarps;
  }
};
template <typename T, int VAR>
struct SmemOp {
  static size_t run() { return VariantKernel<T, VAR>::smem(); }
};
template <typename T, int VAR>
struct LaunchOp {
  static int run(const FusedPlan& pl, const FusedParams<T>& p, cudaStream_t s) {
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
int fused_resident_warps(int device, int variant) {
  return with_variant<T, ResidentOp, int>(variant, device);
}

template <typename T>
FusedPlan plan_fused(int nx, int ny, int variant, int resident_warps, int min_seg) {
  FusedPlan pl;
  pl.variant = variant < 0 || variant >= kVariants ? 0 : variant;
  pl.lanes = fused_variant_lanes<T>(pl.variant);
  const int out = strip_cols(pl.lanes);
  pl.nstrips = (nx + out - 1) / out;
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
  pl.smem = with_variant<T, SmemOp, size_t>(pl.variant);
  return pl;
}

template <typename T>
cudaError_t launch_fused_step(const T* src, T* dst, int nx, int ny, long long pitch,
                              long long plane, const StepConsts<T>& c, int far_rot,
                              const FusedPlan& plan, cudaStream_t s) {
  FusedParams<T> p;
  p.g = march::GridRef<T>{src, dst, nx, ny, pitch, plane, far_rot};
  p.nstrips = plan.nstrips;
  p.seg_len = plan.seg_len;
  p.ntasks = plan.ntasks;
  p.c = c;
  with_variant<T, LaunchOp, int>(plan.variant, plan, p, s);
  return cudaGetLastError();
}

#define LE2D_INST(T)                                                                            \
  template int fused_variant_count<T>();                                                        \
  template int fused_variant_lanes<T>(int);                                                     \
  template int fused_resident_warps<T>(int, int);                                               \
  template FusedPlan plan_fused<T>(int, int, int, int, int);                                    \
  template cudaError_t launch_fused_step<T>(const T*, T*, int, int, long long, long long,       \
                                            const StepConsts<T>&, int, const FusedPlan&,        \
                                            cudaStream_t);
LE2D_INST(float)
LE2D_INST(double)
#undef LE2D_INST

}  // namespace le2d
