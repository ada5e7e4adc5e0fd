// Batched persistent step kernel: many independent solves of different sizes,
// materials and step counts advance together in one launch.
//
// Work list.  Every instance is cut into tiles (strip x row segment, one warp each,
// marched by the same body as the single-solve kernel, march.cuh).  A launch covers
// a window of steps; the work items are (window step r, tile) in step-major order,
// where the tiles of step r are a prefix of the tile list (instances are ordered by
// their step count in the window, longest first).  Warps claim items with one atomic
// counter and loop until the list is empty.
//
// Dependencies instead of grid barriers.  Tile t at step r reads the state its 3x3
// neighbourhood of tiles wrote at step r-1 (2 halo rows, 2 halo columns), and writes
// the buffer those tiles read at step r-1.  So before item (r, t) the warp waits until
// done[n] >= r for every neighbour n (and t itself); after the tile it publishes
// done[t] = r + 1 with release semantics.  Items are claimed in order and a claimed
// item only waits on items of smaller index, all held by running warps, so the
// smallest unfinished item can always proceed.  Every wait is bounded.  A dependency
// wait that runs out (after `wait_ns` of global time) marks its instance failed (the
// instance's failure word) and the warp moves on; every later item of that instance --
// the only items that depend on the missing tile -- is skipped, so the other instances
// of the launch finish normally.  A wait between the two warps of a pair that runs out
// sets ctl->status and ends the launch.  The host reads both (LE2D_ETIMEOUT for the
// failed instances, or for all), the context stays usable.  State loads use
// ld.global.cg: other warps of this launch write them.
//
// FP32 items advance two steps (temporal blocking) on a producer / consumer warp pair
// (march_pair.cuh): the producer claims the item, passes its index to the consumer through
// the pair's queue, waits for the item's dependencies, reads the state and runs the first
// step; the consumer runs the second step on the rows it is handed, writes them, records
// receiver samples and publishes the tile.  The last item of an odd step count, and every
// item of an le_step_soa instance, advances one step: the consumer writes the producer's
// rows as they are.
// A producer may claim its next item while its consumer still finishes the last one: all
// rows of that item are already in the queue, so the consumer finishes without it.
// The x-sweep runs one invariant at a time (sweep_x_lane_diff), which at this kernel's
// occupancy is faster than the packed form the single-solve kernels use; both give the
// same bits.
#include <type_traits>

#include "march_pair.cuh"

namespace le2d {

namespace {

constexpr int kWarps = 4;
constexpr int kNpf = 2;  // input-ring depth of the march (one row in flight ahead)

__device__ __forceinline__ int ld_acquire(const int* p) {
  int v;
  asm volatile("ld.acquire.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_release(int* p, int v) {
  asm volatile("st.release.gpu.global.s32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// True (warp-uniformly) if the instance has failed or the launch is ending.
__device__ __forceinline__ bool instance_off(const int* fail, const BatchCtl* ctl) {
  int off = 0;
  if ((threadIdx.x & 31) == 0)
    off = *reinterpret_cast<const volatile int*>(fail) != 0 ||
          *reinterpret_cast<const volatile int*>(&ctl->status) != 0;
  return __shfl_sync(0xffffffffu, off, 0) != 0;
}

// Waits until every tile of the 3x3 neighbourhood of (seg, strip) has done[] >= r.
// Lanes 0..8 each watch one neighbour.  Returns false if the item is to be skipped: the
// wait gave up (the instance is marked failed), the instance failed meanwhile, or the
// launch is ending (ctl->status).
__device__ __forceinline__ bool wait_neighbours(const int* done, int tile_base, int nstrips,
                                                int nsegs, int seg, int strip, int r, int* fail,
                                                BatchCtl* ctl, unsigned long long wait_ns) {
  const int lane = threadIdx.x & 31;
  const int ds = lane / 3 - 1, dk = lane % 3 - 1;
  const int s2 = seg + ds, k2 = strip + dk;
  const bool watch = lane < 9 && s2 >= 0 && s2 < nsegs && k2 >= 0 && k2 < nstrips;
  const int* p = done + tile_base + (watch ? s2 * nstrips + k2 : 0);
  const unsigned long long t0 = global_ns();
  unsigned ns = 32;
  // gives up after wait_ns of global time over at least 1024 polls (a preempted block sees
  // the clock run on without polling)
  for (unsigned polls = 0;; ++polls) {
    const bool ready = !watch || ld_acquire(p) >= r;
    if (__all_sync(0xffffffffu, ready)) return true;
    int bail = 0;
    if (lane == 0) {
      bail = *reinterpret_cast<volatile int*>(fail) != 0 ||
             *reinterpret_cast<volatile int*>(&ctl->status) != 0;
      if (!bail && polls >= 1024 && global_ns() - t0 > wait_ns) {
        if (atomicExch(fail, 1) == 0) atomicAdd(&ctl->failed, 1);
        bail = 1;
      }
    }
    if (__shfl_sync(0xffffffffu, bail, 0)) return false;
    __nanosleep(ns);
    if (ns < 1024) ns *= 2;
  }
}

// Whether the item of instance I at window step r may run (its dependencies are done).
template <typename T>
__device__ __forceinline__ bool item_ready(const BatchInst<T>& I, const BatchTile& bt, int r,
                                           const int* done, BatchCtl* ctl,
                                           unsigned long long wait_ns) {
  if (r == 0) return !instance_off(I.fail, ctl);
  return wait_neighbours(done, I.tile_base, I.nstrips, I.nsegs, bt.seg, bt.strip, r, I.fail, ctl,
                         wait_ns);
}

__device__ __forceinline__ bool launch_ending(const BatchCtl* ctl) {
  return *reinterpret_cast<const volatile int*>(&ctl->status) != 0;
}

// The one-step kernel's counterpart: the item's step constants in the warp's slot.
template <typename T>
__device__ __forceinline__ const StepConsts<T>& load_step_consts(StepConsts<T>* slot, const StepConsts<T>& c) {
  constexpr int kw = (int)(sizeof(StepConsts<T>) / 4);
  const unsigned* src = reinterpret_cast<const unsigned*>(&c);
  unsigned* dst = reinterpret_cast<unsigned*>(slot);
  for (int i = threadIdx.x & 31; i < kw; i += 32) dst[i] = src[i];
  __syncwarp();
  return *slot;
}

template <typename T, int V, int MINB>
__global__ void __launch_bounds__(kWarps * 32, MINB)
    batch_kernel(const BatchInst<T>* __restrict__ insts, const BatchTile* __restrict__ tiles,
                 const long long* __restrict__ step_items, int nsteps, int* done, BatchCtl* ctl,
                 unsigned long long wait_ns, int stall_plus1) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int lane = threadIdx.x & 31;
  T* ring = reinterpret_cast<T*>(smem_raw) + (threadIdx.x >> 5) * march::warp_smem_elems<T, V, kNpf>();
  StepConsts<T>* cslot = reinterpret_cast<StepConsts<T>*>(
                             smem_raw + kWarps * march::warp_smem_elems<T, V, kNpf>() * sizeof(T)) +
                         (threadIdx.x >> 5);
  const long long total = step_items[nsteps];
  int r = 0;
  while (true) {
    unsigned long long q = 0;
    if (lane == 0) q = atomicAdd(&ctl->next, 1ULL);
    q = __shfl_sync(0xffffffffu, q, 0);
    if ((long long)q >= total) break;
    while ((long long)q >= step_items[r + 1]) ++r;
    const BatchTile bt = tiles[q - step_items[r]];
    const BatchInst<T>& I = insts[bt.inst];
    if (!item_ready(I, bt, r, done, ctl, wait_ns)) {  // the instance failed: skip the item
      if (launch_ending(ctl)) break;
      continue;
    }
    const int par = (I.parity + r) & 1;
    const march::GridRef<T> g{I.buf[par], I.buf[par ^ 1], I.nx, I.ny, I.pitch, I.plane, I.far_rot};
    const int y0 = bt.seg * I.seg_len;
    const int y1 = min(y0 + I.seg_len, I.ny);
    march::RowTap<T> tap{nullptr, -1};
    const long long step_after = I.abs_step0 + r + 1;  // absolute step count after this step
    if (I.trace != nullptr && step_after % I.trace_every == 0)
      tap = march::RowTap<T>{I.trace + (step_after / I.trace_every - 1) * 2 * I.pitch, I.trace_row};
    march::march_tile<T, V, kNpf, true, true, false>(g, load_step_consts(cslot, I.c), bt.strip, y0, y1, ring,
                                                     tap);
    __syncwarp();
    const int tile_id = I.tile_base + bt.seg * I.nstrips + bt.strip;
    if (lane == 0 && !(r == 0 && tile_id == stall_plus1 - 1)) {
      __threadfence();
      st_release(done + tile_id, r + 1);
    }
  }
}

// The sweep constants of the item a warp of a pair works on, copied from the instance record
// into the warp's own slot of shared memory when it starts the item: the march reads them
// every row, and the record lives in global memory (the single-solve kernels take them from
// the kernel parameters instead).  The y-sweep's come as the pairs the packed y-pipeline
// multiplies by.
template <typename T>
struct ItemConsts {
  Sweep<T> x;
  YPairs y;
};
template <typename T>
__host__ __device__ constexpr int item_consts_bytes() { return ((int)sizeof(ItemConsts<T>) + 15) / 16 * 16; }

// Shared memory of one pair of the batched kernel: the march's, then one ItemConsts slot
// per warp.
template <typename T, int V>
__host__ __device__ constexpr int batch_pair_bytes() { return march::pair_smem_bytes<T, V, kNpf>() + 2 * item_consts_bytes<T>(); }

template <typename T>
__device__ __forceinline__ const ItemConsts<T>& load_item_consts(ItemConsts<T>* slot, const BatchInst<T>& I) {
  constexpr int kx = (int)(sizeof(Sweep<T>) / 4), ky = (int)(sizeof(YPairs) / 4);
  const int lane = threadIdx.x & 31;
  const unsigned* sx = reinterpret_cast<const unsigned*>(&I.c.x);
  const unsigned* sy = reinterpret_cast<const unsigned*>(&I.yq);
  unsigned* dx = reinterpret_cast<unsigned*>(&slot->x);
  unsigned* dy = reinterpret_cast<unsigned*>(&slot->y);
  for (int i = lane; i < kx; i += 32) dx[i] = sx[i];
  for (int i = lane; i < ky; i += 32) dy[i] = sy[i];
  __syncwarp();
  return *slot;
}

template <typename T, int V, int MINB>
__global__ void __launch_bounds__(kWarps * 32, MINB)
    batch_pair_kernel(const BatchInst<T>* __restrict__ insts, const BatchTile* __restrict__ tiles,
                      const long long* __restrict__ step_items, int nsteps, int* done,
                      BatchCtl* ctl, unsigned long long wait_ns, int stall_plus1) {
  using march::kHand;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int lane = threadIdx.x & 31;
  const int wib = threadIdx.x >> 5;
  const bool producer = (wib & 1) == 0;
  unsigned char* base = smem_raw + (wib >> 1) * batch_pair_bytes<T, V>();
  T* smem = reinterpret_cast<T*>(base);
  ItemConsts<T>* kslot = reinterpret_cast<ItemConsts<T>*>(base + march::pair_smem_bytes<T, V, kNpf>() +
                                                          (wib & 1) * item_consts_bytes<T>());
  unsigned long long* bars =
      reinterpret_cast<unsigned long long*>(base + march::pair_smem_elems<T, V, kNpf>() * sizeof(T));
  volatile long long* item_q = reinterpret_cast<volatile long long*>(bars + 2 * kHand);
  if (producer) march::pair_init<T, V>(bars);
  __syncthreads();
  const long long total = step_items[nsteps];
  int* status = &ctl->status;
  unsigned u = 0;  // handoffs through the pair's queue (item indices and rows)
  int r = 0;
  // The two roles run separate loops (each keeps only its own state live across its march).
  if (producer) {
    while (true) {
      unsigned long long claimed = 0;
      if (lane == 0) claimed = atomicAdd(&ctl->next, 1ULL);
      const long long q = (long long)__shfl_sync(0xffffffffu, claimed, 0);
      // the item's dependencies first, then the hand-off: a skipped item (its instance
      // failed) goes to the consumer as -(q + 1)
      bool skip = false;
      if (q < total) {
        while (q >= step_items[r + 1]) ++r;
        const BatchTile bt = tiles[q - step_items[r]];
        skip = !item_ready(insts[bt.inst], bt, r, done, ctl, wait_ns);
        if (skip && launch_ending(ctl)) break;
      }
      const int hs = (int)(u % kHand);
      const unsigned use = u / kHand;
      if (use > 0 && !march::mbar_wait(bars + kHand + hs, (use - 1) & 1, wait_ns, status)) break;
      if (lane == 0) item_q[hs] = skip ? -(q + 1) : q;
      march::mbar_arrive(bars + hs);
      ++u;
      if (q >= total) break;
      if (skip) continue;
      const BatchTile bt = tiles[q - step_items[r]];
      const BatchInst<T>& I = insts[bt.inst];
      const int nadv = min(I.depth, I.steps - r * I.depth);  // steps this item advances
      const int par = (I.parity + r) & 1;
      const march::GridRef<T> g{I.buf[par], I.buf[par ^ 1], I.nx, I.ny, I.pitch, I.plane, I.far_rot};
      const int y0 = bt.seg * I.seg_len;
      const int y1 = min(y0 + I.seg_len, I.ny);
      const ItemConsts<T>& k = load_item_consts(kslot, I);
      if (!march::pair_produce<T, V, kNpf, true, false>(g, k.x, k.y, bt.strip, y0, y1, smem, bars, wait_ns,
                                                        status, u, nadv == 1))
        break;
    }
  } else {
    // the producer hands over an item only after its dependency wait, which may run out
    // (wait_ns) and hand over a skip instead: the consumer's wait for the item outlasts it
    const unsigned long long item_wait_ns = wait_ns > ~0ULL / 4 ? ~0ULL : 4 * wait_ns;
    while (true) {
      const int hs = (int)(u % kHand);
      if (!march::mbar_wait(bars + hs, (u / kHand) & 1, item_wait_ns, status)) break;
      const long long q = item_q[hs];
      march::mbar_arrive(bars + kHand + hs);
      ++u;
      if (q < 0) continue;  // skipped by the producer: its instance failed
      if (q >= total) break;
      while (q >= step_items[r + 1]) ++r;
      const BatchTile bt = tiles[q - step_items[r]];
      const BatchInst<T>& I = insts[bt.inst];
      const int nadv = min(I.depth, I.steps - r * I.depth);
      const int par = (I.parity + r) & 1;
      const march::GridRef<T> g{I.buf[par], I.buf[par ^ 1], I.nx, I.ny, I.pitch, I.plane, I.far_rot};
      const int y0 = bt.seg * I.seg_len;
      const int y1 = min(y0 + I.seg_len, I.ny);
      // receiver samples after the item's first and (two-step items) second step
      const long long before = I.abs_step0 + (long long)r * I.depth;
      march::RowTap<T> tap_a{nullptr, -1}, tap_b{nullptr, -1};
      if (I.trace != nullptr && (before + 1) % I.trace_every == 0)
        tap_a = march::RowTap<T>{I.trace + ((before + 1) / I.trace_every - 1) * 2 * I.pitch, I.trace_row};
      if (I.trace != nullptr && nadv == 2 && (before + 2) % I.trace_every == 0)
        tap_b = march::RowTap<T>{I.trace + ((before + 2) / I.trace_every - 1) * 2 * I.pitch, I.trace_row};
      const int tile_id = I.tile_base + bt.seg * I.nstrips + bt.strip;
      const ItemConsts<T>& k = load_item_consts(kslot, I);
      if (!march::pair_consume<T, V, kNpf, true, false>(g, k.x, k.y, bt.strip, y0, y1, smem, bars, wait_ns,
                                                        status, u, nadv == 1, tap_a, tap_b))
        break;
      __syncwarp();  // the consumer wrote the tile's new state and publishes it
      if (lane == 0 && !(r == 0 && tile_id == stall_plus1 - 1)) {
        __threadfence();
        st_release(done + tile_id, r + 1);
      }
    }
  }
}

template <typename T>
struct BatchKernelOf;
// FP32: two-step items on warp pairs (4 columns per lane, 168 registers: 12 warps per SM);
// FP64: one-step items on single warps (2 columns per lane, 8 warps per SM); each warp's
// ring is followed, after all the block's rings, by its step-constants slot.
template <>
struct BatchKernelOf<float> {
  static constexpr int V = 4, MINB = 3, DEPTH = 2;
  static void* fn() { return (void*)batch_pair_kernel<float, V, MINB>; }
  static size_t smem() { return (size_t)(kWarps / 2) * batch_pair_bytes<float, V>(); }
};
static_assert(march::warp_smem_elems<double, 2, kNpf>() * sizeof(double) % alignof(StepConsts<double>) == 0,
              "the step-constants slots after the rings must stay aligned");
template <>
struct BatchKernelOf<double> {
  static constexpr int V = 2, MINB = 2, DEPTH = 1;
  static void* fn() { return (void*)batch_kernel<double, V, MINB>; }
  static size_t smem() {
    return (size_t)kWarps * (march::warp_smem_elems<double, V, kNpf>() * sizeof(double) + sizeof(StepConsts<double>));
  }
};

}  // namespace

template <typename T>
int batch_lanes() { return BatchKernelOf<T>::V; }

template <typename T>
int batch_depth() { return BatchKernelOf<T>::DEPTH; }

template <typename T>
size_t batch_smem() { return BatchKernelOf<T>::smem(); }

template <typename T>
int batch_resident_blocks(int device) {
  using K = BatchKernelOf<T>;
  int sms = 0, per_sm = 0;
  // dynamic shared memory above 48 KB is opted into once (before any launch or capture)
  cudaFuncSetAttribute(K::fn(), cudaFuncAttributeMaxDynamicSharedMemorySize, (int)batch_smem<T>());
  if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device) != cudaSuccess) return 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, K::fn(), kWarps * 32, batch_smem<T>()) !=
      cudaSuccess)
    return 0;
  return sms * per_sm;
}

template <typename T>
cudaError_t launch_batch(const BatchInst<T>* insts, const BatchTile* tiles,
                         const long long* step_items, int nsteps, long long total_items, int* done,
                         BatchCtl* ctl, unsigned long long wait_ns, int stall_plus1,
                         int resident_blocks, cudaStream_t s) {
  using K = BatchKernelOf<T>;
  const int per_block = K::DEPTH == 2 ? kWarps / 2 : kWarps;  // items a block works on at once
  long long blocks = (total_items + per_block - 1) / per_block;
  if (blocks > resident_blocks) blocks = resident_blocks;  // persistent: all blocks resident
  if (blocks < 1) blocks = 1;
  if constexpr (K::DEPTH == 2)
    batch_pair_kernel<T, K::V, K::MINB><<<(int)blocks, kWarps * 32, batch_smem<T>(), s>>>(
        insts, tiles, step_items, nsteps, done, ctl, wait_ns, stall_plus1);
  else
    batch_kernel<T, K::V, K::MINB><<<(int)blocks, kWarps * 32, batch_smem<T>(), s>>>(
        insts, tiles, step_items, nsteps, done, ctl, wait_ns, stall_plus1);
  return cudaGetLastError();
}

#ifdef LE2D_CHECK
unsigned long long check_violations_batch() {
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
  template int batch_lanes<T>();                                                                \
  template int batch_depth<T>();                                                                \
  template size_t batch_smem<T>();                                                              \
  template int batch_resident_blocks<T>(int);                                                   \
  template cudaError_t launch_batch<T>(const BatchInst<T>*, const BatchTile*, const long long*, \
                                       int, long long, int*, BatchCtl*, unsigned long long, int, \
                                       int, cudaStream_t);
LE2D_INST(float)
LE2D_INST(double)
#undef LE2D_INST

}  // namespace le2d
