// Two time steps per launch on a warp pair.  The tile's first step (step A) and second
// step (step B) run on two warps of one block: the producer warp reads the state, x-sweeps
// and y-sweeps it (step A) and hands each finished row to the consumer warp through a
// small shared-memory queue; the consumer x-sweeps and y-sweeps those rows (step B) and
// writes the result.  Each warp holds one y-pipeline, so four columns per lane fit in
// 128 registers and 16 warps per SM, where one warp holding both steps needs twice the
// pipeline state (march2.cuh).
//
// Queue.  kHand slots of one row (5 fields x 32V columns), each with two mbarriers of
// arrival count 32: `full` (every producer lane arrives after writing its columns) and
// `empty` (every consumer lane arrives after reading its columns).  The u-th handoff
// uses slot u % kHand, its (u / kHand)-th use: the consumer waits for phase u / kHand of
// `full`, the producer (from the second use of a slot on) for phase u / kHand - 1 of
// `empty`.  Each lane reads back exactly the columns the same lane of the other warp wrote.
//
// Every wait is bounded (wait_ns of global time over at least kMinPolls polls); a warp that
// gives up sets *status and leaves, so its partner gives up too and the launch ends with
// the status set.
//
// Halos and boundaries as in march2.cuh: step A is valid on [xs+2, xs+32V-2), step B on
// [xs+4, xs+32V-4); the producer overwrites step A's values outside [0, nx) with the edge
// column's and hands row 0 / ny-1 over once and the consumer feeds it to step B once for
// every row of its stencil it stands for (the same count both warps compute).  A one-step
// tile (in the batched kernel: an odd last step, or le_step_soa's far end) hands over step
// A's own rows [y0, y1), which the consumer writes as they are.
#pragma once

#include "march2.cuh"

namespace le2d {
namespace march {

constexpr int kHand = 1;  // queue slots between the warps of a pair

__device__ __forceinline__ unsigned smem_u32(const void* p) {
  return (unsigned)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void mbar_init(unsigned long long* bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_arrive(unsigned long long* bar) {
  asm volatile("{\n\t.reg .b64 st;\n\tmbarrier.arrive.shared::cta.b64 st, [%0];\n\t}" ::"r"(smem_u32(bar))
               : "memory");
}
// Tests for the completion of the phase with parity `parity`; while it is incomplete the
// thread is suspended (it issues nothing) until the phase completes or about 0.5 ms pass.
__device__ __forceinline__ bool mbar_test(unsigned long long* bar, unsigned parity) {
  unsigned ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity), "r"(500000u)
      : "memory");
  return ok != 0;
}
__device__ __forceinline__ unsigned long long global_timer_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// Waits (all 32 lanes) for the completion of the phase of `bar` with parity `parity`.
// Returns false, warp-uniformly, once it has waited more than wait_ns of global time over
// at least kMinPolls polls, or as soon as the partner has given up (*status != 0).  Both
// bounds must pass: a block that another context preempts sees the clock run on without
// polling, and a poll that returns at once takes no time.
constexpr unsigned kMinPolls = 1024;
static __device__ __noinline__ bool mbar_wait_slow(unsigned long long* bar, unsigned parity, bool ok,
                                                   unsigned long long wait_ns, int* status) {
  const unsigned long long t0 = global_timer_ns();
  for (unsigned polls = 1;; ++polls) {
    if (!ok) ok = mbar_test(bar, parity);
    if (__all_sync(0xffffffffu, ok)) return true;
    int bail = 0;
    if ((threadIdx.x & 31) == 0)
      bail = *reinterpret_cast<volatile int*>(status) != 0 ||
             (polls >= kMinPolls && global_timer_ns() - t0 > wait_ns);
    if (__shfl_sync(0xffffffffu, bail, 0)) {
      if ((threadIdx.x & 31) == 0) atomicExch(status, 1);
      return false;
    }
  }
}
// The first test inline; the polling loop is a call, which keeps it out of the loops that
// wait once per row (their code has to stay small enough for the instruction cache).
__device__ __forceinline__ bool mbar_wait(unsigned long long* bar, unsigned parity,
                                          unsigned long long wait_ns, int* status) {
  const bool ok = mbar_test(bar, parity);
  if (__all_sync(0xffffffffu, ok)) return true;
  return mbar_wait_slow(bar, parity, ok, wait_ns, status);
}

// Shared memory of one pair: the producer's input ring (NPF rows) and step-A ring (3),
// the queue (kHand), the consumer's step-B ring (3), each row NF x 32V elements; then
// 2 * kHand mbarriers and kHand 8-byte words a persistent kernel passes work items in.
template <typename T, int V, int NPF>
__host__ __device__ constexpr int pair_smem_elems() {
  return (NPF + 3 + kHand + 3) * NF * 32 * V;
}
// Rounded up to 16 bytes: the next pair of the block starts where this one ends, and its
// rows are read and written with 16-byte vector accesses.
template <typename T, int V, int NPF>
__host__ __device__ constexpr int pair_smem_bytes() {
  return (pair_smem_elems<T, V, NPF>() * (int)sizeof(T) + 2 * kHand * 8 + kHand * 8 + 15) / 16 * 16;
}
static_assert(pair_smem_bytes<float, 4, 2>() % 16 == 0 && pair_smem_bytes<double, 2, 3>() % 16 == 0,
              "pair shared memory must keep 16-byte alignment");

// How many rows of step B's stencil step-A row ka stands for (tile rows [y0, y1)):
// step B reads rows [y0-2, y1+2) clamped to [0, ny).  A one-step tile hands over its own
// rows [y0, y1) only, once each.
__device__ __forceinline__ int row_uses(int ka, int y0, int y1, int ny, bool one_step = false) {
  if (one_step) return ka >= y0 && ka < y1 ? 1 : 0;
  int reps = ka < 0 || ka >= ny ? 0 : 1;
  if (ka == 0 && y0 < 2) reps += 2 - y0;
  if (ka == ny - 1 && y1 + 2 > ny) reps += y1 + 2 - ny;
  return reps;
}

template <typename T, int V>
__device__ __forceinline__ void pair_init(unsigned long long* bars) {
  if ((threadIdx.x & 31) == 0)
    for (int i = 0; i < 2 * kHand; ++i) mbar_init(bars + i, 32);
}

// Writes vx and vy of a row into a receiver line (RowTap) for this lane's V columns.
template <typename T, int V>
__device__ __forceinline__ void tap_row(const RowTap<T>& tap, long long pitch, int col0,
                                        const T (&f)[NF][V]) {
  using VT = typename Vec<T, V>::type;
  if (!in_line(col0, V, pitch)) return;
  *reinterpret_cast<VT*>(tap.out + col0) = pack(f[VX]);
  *reinterpret_cast<VT*>(tap.out + pitch + col0) = pack(f[VY]);
}

// Interior tiles.  When the strip lies inside [0, nx), every row the tile reads lies inside
// [0, ny) (y0 >= 4, y1 + 4 <= ny) and the tile takes two steps, no column or row is
// clamped and every step-A row ka in [y0-2, y1+2) is handed over exactly once -- the same
// handoffs pair_produce / pair_consume make for such a tile, in the same order.  These
// loops drop the clamps and the per-row use counts, step the row addresses instead of
// recomputing them and store with predicates: about 9 % fewer instructions per node-update
// with a loop no larger than the general one (a loop over two rows, which would let the
// y-pipeline's replaced states alternate instead of being copied, measured slower: it no
// longer fits the instruction cache).  Any input-ring depth NPF >= 2.
template <typename T, int V>
__device__ __forceinline__ bool tile_is_interior(const GridRef<T>& g, int xs, int y0, int y1) {
  return xs >= 0 && xs + 32 * V <= g.nx && y0 >= 4 && y1 + 4 <= g.ny;
}

template <typename T, int V>
__device__ __forceinline__ void fetch_interior(T* slot, const T* row, long long plane) {
  constexpr int kIn = 32 * V;
#pragma unroll
  for (int k = 0; k < NF; ++k) cp_async<V * (int)sizeof(T)>(slot + k * kIn, row + k * plane);
  cp_async_commit();
}
// The bounds-checked build checks each row against the grid (a separate function: handing
// the grid to the unchecked one changes the register allocation of the lean loops).
#ifdef LE2D_CHECK
template <typename T, int V>
__device__ __forceinline__ void fetch_interior_checked(T* slot, const T* row, const GridRef<T>& g) {
  constexpr int kIn = 32 * V;
#pragma unroll
  for (int k = 0; k < NF; ++k)
    if (in_src(g, row + k * g.plane, V)) cp_async<V * (int)sizeof(T)>(slot + k * kIn, row + k * g.plane);
  cp_async_commit();
}
#define LE2D_FETCH_INTERIOR(T, V, slot, row, g) fetch_interior_checked<T, V>(slot, row, g)
#else
#define LE2D_FETCH_INTERIOR(T, V, slot, row, g) fetch_interior<T, V>(slot, row, (g).plane)
#endif

// `cy`: the y-sweep constants (Sweep, or YPairs for the FP32 pipeline).
template <typename T, int V, int NPF, typename CY>
__device__ __forceinline__ bool pair_produce_interior(const GridRef<T>& g, const Sweep<T>& cx,
                                                      const CY& cy, int xs, int y0, int y1,
                                                      T* smem_pair, unsigned long long* bars,
                                                      unsigned long long wait_ns, int* status,
                                                      unsigned& u) {
  using VT = typename Vec<T, V>::type;
  static_assert(NPF >= 2, "the input ring needs at least the current and the next row");
  constexpr int kIn = 32 * V;
  constexpr int kRow = NF * kIn;
  const int lane = threadIdx.x & 31;
  T* in_ring = smem_pair + lane * V;
  T* a_ring = in_ring + NPF * kRow;
  T* hand = a_ring + 3 * kRow;
  unsigned long long* full = bars;
  unsigned long long* empty = bars + kHand;
  const int mend = y1 + 4;

  YPipe<T, V> ya;
  ya.init();
#pragma unroll
  for (int k = 0; k < NF; ++k) *reinterpret_cast<VT*>(a_ring + 2 * kRow + k * kIn) = VT{};
  const T* next = g.src + (long long)(y0 - 4) * g.pitch + xs + lane * V;  // next row to fetch
#pragma unroll
  for (int j = 0; j < NPF - 1; ++j) {
    LE2D_FETCH_INTERIOR(T, V, in_ring + j * kRow, next, g);
    next += g.pitch;
  }
  int aslot = 0;
  int islot = 0;  // input slot of row m; row m+NPF-1 goes to the slot before it
  bool ok = true;
  for (int m = y0 - 4; m < mend; ++m) {
    if (m + NPF - 1 < mend) {
      LE2D_FETCH_INTERIOR(T, V, in_ring + (islot == 0 ? NPF - 1 : islot - 1) * kRow, next, g);
      next += g.pitch;
    } else {
      cp_async_commit();  // keep one group per row
    }
    cp_async_wait<NPF - 1>();
    T f[NF][V];
#pragma unroll
    for (int k = 0; k < NF; ++k) unpack(*reinterpret_cast<const VT*>(in_ring + islot * kRow + k * kIn), f[k]);
    sweep_x_lane<T, V>(f, cx);
    ring_left(ya, f, a_ring, aslot, cy);
    if (m >= y0) {  // step-A row m-2 is complete and handed over
      T ga[NF][V];
      ring_output(ya, ga, a_ring, aslot, cy);
      const int hs = (int)(u % kHand);
      const unsigned use = u / kHand;
      if (use > 0 && !mbar_wait(empty + hs, (use - 1) & 1, wait_ns, status)) {
        ok = false;
        break;
      }
      T* slot = hand + hs * kRow;
#pragma unroll
      for (int k = 0; k < NF; ++k) *reinterpret_cast<VT*>(slot + k * kIn) = pack(ga[k]);
      mbar_arrive(full + hs);
      ++u;
    }
    ya.right(cy);
    islot = islot + 1 == NPF ? 0 : islot + 1;
    aslot = aslot == 2 ? 0 : aslot + 1;
  }
  cp_async_wait<0>();  // nothing of this warp's in flight when it leaves (also after a break)
  return ok;
}

template <typename T, int V, int NPF, typename CY>
__device__ __forceinline__ bool pair_consume_interior(const GridRef<T>& g, const Sweep<T>& cx,
                                                      const CY& cy, int xs, int y0, int y1,
                                                      T* smem_pair, unsigned long long* bars,
                                                      unsigned long long wait_ns, int* status,
                                                      unsigned& u) {
  using VT = typename Vec<T, V>::type;
  constexpr int H2 = halo_lanes2(V);
  constexpr int kIn = 32 * V;
  constexpr int kRow = NF * kIn;
  const int lane = threadIdx.x & 31;
  T* hand = smem_pair + lane * V + (NPF + 3) * kRow;
  T* b_ring = hand + kHand * kRow;
  unsigned long long* full = bars;
  unsigned long long* empty = bars + kHand;
  const bool writer = lane >= H2 && lane < 32 - H2;

  YPipe<T, V> yb;
  yb.init();
#pragma unroll
  for (int k = 0; k < NF; ++k) *reinterpret_cast<VT*>(b_ring + 2 * kRow + k * kIn) = VT{};
  T* out = g.dst + (long long)y0 * g.pitch + xs + lane * V;  // next row written
  int bslot = 0;
  for (int ka = y0 - 2; ka < y1 + 2; ++ka) {
    const int hs = (int)(u % kHand);
    if (!mbar_wait(full + hs, (u / kHand) & 1, wait_ns, status)) return false;
    const T* slot = hand + hs * kRow;
    T fb[NF][V];
#pragma unroll
    for (int k = 0; k < NF; ++k) unpack(*reinterpret_cast<const VT*>(slot + k * kIn), fb[k]);
    mbar_arrive(empty + hs);
    sweep_x_lane<T, V>(fb, cx);
    ring_left(yb, fb, b_ring, bslot, cy);
    if (ka >= y0 + 2) {  // step-B row ka-2 is complete
      T gb[NF][V];
      ring_output(yb, gb, b_ring, bslot, cy);
#pragma unroll
      for (int k = 0; k < NF; ++k) store_if(writer && in_dst(g, out + k * g.plane, V), reinterpret_cast<VT*>(out + k * g.plane), pack(gb[k]));
      out += g.pitch;
    }
    yb.right(cy);
    bslot = bslot == 2 ? 0 : bslot + 1;
    ++u;
  }
  return true;
}

// One step on one warp (march_tile) for an interior tile of a one-step launch: the strip
// inside [0, nx) and the rows [y0-2, y1+2) it reads inside [0, ny), so no clamps, row
// addresses stepped, predicated stores.
template <typename T, int V>
__device__ __forceinline__ bool tile_is_interior1(const GridRef<T>& g, int xs, int y0, int y1) {
  return xs >= 0 && xs + 32 * V <= g.nx && y0 >= 2 && y1 + 2 <= g.ny;
}

template <typename T, int V, int NPF>
__device__ __forceinline__ void march_tile_interior(const GridRef<T>& g, const StepConsts<T>& c, int xs,
                                                    int y0, int y1, T* smem_warp) {
  using VT = typename Vec<T, V>::type;
  static_assert(NPF >= 2, "the input ring needs at least the current and the next row");
  constexpr int H = halo_lanes(V);
  constexpr int kIn = 32 * V;
  constexpr int kRow = NF * kIn;
  const int lane = threadIdx.x & 31;
  T* in_ring = smem_warp + lane * V;
  T* xs_ring = in_ring + NPF * kRow;
  const bool writer = lane >= H && lane < 32 - H;
  const int mend = y1 + 2;

  YPipe<T, V> yp;
  yp.init();
#pragma unroll
  for (int k = 0; k < NF; ++k) *reinterpret_cast<VT*>(xs_ring + 2 * kRow + k * kIn) = VT{};
  const T* next = g.src + (long long)(y0 - 2) * g.pitch + xs + lane * V;  // next row to fetch
#pragma unroll
  for (int j = 0; j < NPF - 1; ++j) {
    LE2D_FETCH_INTERIOR(T, V, in_ring + j * kRow, next, g);
    next += g.pitch;
  }
  T* out = g.dst + (long long)y0 * g.pitch + xs + lane * V;  // next row written
  int islot = 0, xslot = 0;
  for (int m = y0 - 2; m < mend; ++m) {
    if (m + NPF - 1 < mend) {
      LE2D_FETCH_INTERIOR(T, V, in_ring + (islot == 0 ? NPF - 1 : islot - 1) * kRow, next, g);
      next += g.pitch;
    } else {
      cp_async_commit();  // keep one group per row
    }
    cp_async_wait<NPF - 1>();
    T f[NF][V];
#pragma unroll
    for (int k = 0; k < NF; ++k) unpack(*reinterpret_cast<const VT*>(in_ring + islot * kRow + k * kIn), f[k]);
    sweep_x_lane<T, V>(f, c.x);
    ring_left(yp, f, xs_ring, xslot, c.y);
    if (m >= y0 + 2) {  // row m-2 is complete
      T gf[NF][V];
      ring_output(yp, gf, xs_ring, xslot, c.y);
#pragma unroll
      for (int k = 0; k < NF; ++k) store_if(writer && in_dst(g, out + k * g.plane, V), reinterpret_cast<VT*>(out + k * g.plane), pack(gf[k]));
      out += g.pitch;
    }
    yp.right(c.y);
    islot = islot + 1 == NPF ? 0 : islot + 1;
    xslot = xslot == 2 ? 0 : xslot + 1;
  }
}

// Producer warp: step A of strip `strip`, rows [y0, y1) of the tile, handing its rows to
// the consumer; `u` counts the queue's handoffs (it continues across tiles).  A one_step
// tile (an odd last step, or le_step_soa's far end, which g.far_rot selects) hands over
// step A's rows [y0, y1) only, which the consumer writes.  Returns false if a wait gave up.
template <typename T, int V, int NPF, bool COHERENT, bool XPACK = true, typename CY = Sweep<T>>
__device__ __forceinline__ bool pair_produce(const GridRef<T>& g, const Sweep<T>& cx, const CY& cy, int strip,
                                             int y0, int y1, T* smem_pair,
                                             unsigned long long* bars,
                                             unsigned long long wait_ns, int* status, unsigned& u,
                                             bool one_step) {
  using VT = typename Vec<T, V>::type;
  static_assert(NPF >= 2, "the input ring needs at least the current and the next row");
  static_assert(!COHERENT || V * sizeof(T) == 16, "coherent loads need 16-byte (L2-only) copies");
  constexpr int H2 = halo_lanes2(V);
  constexpr int kIn = 32 * V;
  constexpr int kOut = strip_cols2(V);
  constexpr int kRow = NF * kIn;
  const int lane = threadIdx.x & 31;
  T* in_ring = smem_pair + lane * V;
  T* a_ring = in_ring + NPF * kRow;
  T* hand = a_ring + 3 * kRow;
  unsigned long long* full = bars;
  unsigned long long* empty = bars + kHand;
  const int xs = strip * kOut - H2 * V;
  const int col0 = xs + lane * V;
  const bool interior = xs >= 0 && xs + kIn <= g.nx;
  const int mend = one_step ? y1 + 2 : y1 + 4;  // one step needs the raw rows up to y1+1 only

  YPipe<T, V> ya;
  ya.init();
#pragma unroll
  for (int k = 0; k < NF; ++k) *reinterpret_cast<VT*>(a_ring + 2 * kRow + k * kIn) = VT{};
#pragma unroll
  for (int j = 0; j < NPF - 1; ++j)
    fetch_row<T, V, COHERENT>(in_ring + j * kRow, g, source_row(y0 - 4 + j, g.ny, g.far_rot), col0,
                              interior);
  int islot = 0, aslot = 0;
  bool ok = true;
  for (int m = y0 - 4; m < mend; ++m) {
    {
      const int mm = m + NPF - 1;
      const int ns = islot + NPF - 1 >= NPF ? islot - 1 : islot + NPF - 1;
      if (mm < mend)
        fetch_row<T, V, COHERENT>(in_ring + ns * kRow, g, source_row(mm, g.ny, g.far_rot), col0,
                                  interior);
      else
        cp_async_commit();
    }
    cp_async_wait<NPF - 1>();
    T f[NF][V];
#pragma unroll
    for (int k = 0; k < NF; ++k)
      unpack(*reinterpret_cast<const VT*>(in_ring + islot * kRow + k * kIn), f[k]);
    if (!interior) clamp_lane<T, V>(f, col0, g.nx);
    sweep_x_lane<T, V, XPACK>(f, cx);
    ring_left(ya, f, a_ring, aslot, cy);
    const int ka = m - 2;  // step-A row completed now
    if (m >= y0 && row_uses(ka, y0, y1, g.ny, one_step) > 0) {
      T ga[NF][V];
      ring_output(ya, ga, a_ring, aslot, cy);
      if (!interior) clamp_columns<T, V>(ga, xs, col0, g.nx);
      const int hs = (int)(u % kHand);
      const unsigned use = u / kHand;
      if (use > 0 && !mbar_wait(empty + hs, (use - 1) & 1, wait_ns, status)) {
        ok = false;
        break;
      }
      T* slot = hand + hs * kRow;
#pragma unroll
      for (int k = 0; k < NF; ++k) *reinterpret_cast<VT*>(slot + k * kIn) = pack(ga[k]);
      mbar_arrive(full + hs);
      ++u;
    }
    ya.right(cy);
    islot = islot + 1 == NPF ? 0 : islot + 1;
    aslot = aslot == 2 ? 0 : aslot + 1;
  }
  cp_async_wait<0>();  // nothing of this warp's in flight when it leaves (also after a break)
  return ok;
}

// Consumer warp: step B of the same tile, writing rows [y0, y1) to g.dst; `u` as for the
// producer.  A one_step tile's handed rows are step A's rows [y0, y1), written as they
// are.  TAP: receiver rows -- tap_a of the rows after step A (taken from the handed rows),
// tap_b of the rows after step B.  Returns false if a wait gave up.
template <typename T, int V, int NPF, bool TAP, bool XPACK = true, typename CY = Sweep<T>>
__device__ __forceinline__ bool pair_consume(const GridRef<T>& g, const Sweep<T>& cx, const CY& cy, int strip,
                                             int y0, int y1, T* smem_pair,
                                             unsigned long long* bars,
                                             unsigned long long wait_ns, int* status, unsigned& u,
                                             bool one_step, const RowTap<T>& tap_a,
                                             const RowTap<T>& tap_b) {
  using VT = typename Vec<T, V>::type;
  constexpr int H2 = halo_lanes2(V);
  constexpr int kIn = 32 * V;
  constexpr int kOut = strip_cols2(V);
  constexpr int kRow = NF * kIn;
  const int lane = threadIdx.x & 31;
  T* hand = smem_pair + lane * V + (NPF + 3) * kRow;
  T* b_ring = hand + kHand * kRow;
  unsigned long long* full = bars;
  unsigned long long* empty = bars + kHand;
  const int xs = strip * kOut - H2 * V;
  const int col0 = xs + lane * V;
  const bool writer = lane >= H2 && lane < 32 - H2 && col0 < g.nx;

  YPipe<T, V> yb;
  yb.init();
#pragma unroll
  for (int k = 0; k < NF; ++k) *reinterpret_cast<VT*>(b_ring + 2 * kRow + k * kIn) = VT{};
  int bslot = 0;
  int bin = y0 - 2;  // step-B row index of the next row fed to step B
  for (int ka = y0 - 2; ka < y1 + 2; ++ka) {
    const int reps = row_uses(ka, y0, y1, g.ny, one_step);
    if (reps == 0) continue;
    const int hs = (int)(u % kHand);
    if (!mbar_wait(full + hs, (u / kHand) & 1, wait_ns, status)) return false;
    const T* slot = hand + hs * kRow;
    if (TAP && ka == tap_a.row && ka >= y0 && ka < y1 && writer) {
      T fa[NF][V];
#pragma unroll
      for (int k = 0; k < NF; ++k) unpack(*reinterpret_cast<const VT*>(slot + k * kIn), fa[k]);
      tap_row<T, V>(tap_a, g.pitch, col0, fa);
    }
    if (one_step) {  // step A's row ka in [y0, y1): written as handed over
      T fa[NF][V];
#pragma unroll
      for (int k = 0; k < NF; ++k) unpack(*reinterpret_cast<const VT*>(slot + k * kIn), fa[k]);
      mbar_arrive(empty + hs);
      T* out = g.dst + (long long)ka * g.pitch + col0;
#pragma unroll
      for (int k = 0; k < NF; ++k) store_if(writer && in_dst(g, out + k * g.plane, V), reinterpret_cast<VT*>(out + k * g.plane), pack(fa[k]));
      ++u;
      continue;
    }
    for (int r = 0; r < reps; ++r) {  // the slot is read once per use, released after the last
      T fb[NF][V];
#pragma unroll
      for (int k = 0; k < NF; ++k) unpack(*reinterpret_cast<const VT*>(slot + k * kIn), fb[k]);
      if (r == reps - 1) mbar_arrive(empty + hs);
      sweep_x_lane<T, V, XPACK>(fb, cx);
      ring_left(yb, fb, b_ring, bslot, cy);
      if (bin >= y0 + 2) {  // step-B row bin-2 is complete
        T gb[NF][V];
        ring_output(yb, gb, b_ring, bslot, cy);
        const int row = bin - 2;
        T* out = g.dst + (long long)row * g.pitch + col0;
#pragma unroll
        for (int k = 0; k < NF; ++k) store_if(writer && in_dst(g, out + k * g.plane, V), reinterpret_cast<VT*>(out + k * g.plane), pack(gb[k]));
        if (TAP && row == tap_b.row && writer) tap_row<T, V>(tap_b, g.pitch, col0, gb);
      }
      yb.right(cy);
      bslot = bslot == 2 ? 0 : bslot + 1;
      ++bin;
    }
    ++u;
  }
  return true;
}

}  // namespace march
}  // namespace le2d
