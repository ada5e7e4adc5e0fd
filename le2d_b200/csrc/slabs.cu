// One grid split into row slabs over several devices (the reference's multi-GPU scheme,
// le2d cuda5/cuda6: le_core.cu:374-509, one process driving every device with peer
// copies of the rows next to each cut; the copies overlapped with the interior, as
// cuda6/le_core.cu:456-482 overlaps them with its y-sweep).
//
// Slab s owns the global rows [r0, r1) and keeps a copy of kHalo rows on each side that
// has a neighbour (none at the grid's top and bottom), so its device grid is the rows
// [r0 - h0, r1 + h1).  A launch advances a slab by up to two steps with the unmodified
// fused kernels, writing only its owned rows: the stencil of two steps reaches 4 rows, so
// the owned rows come out exact from the owned and halo rows of the launch before.
//
// Per launch and slab, in this order of dependencies:
//   band     the owned rows beside each cut (4 each), on a high-priority stream, after
//            the slab's previous interior and the halo copies into the slab;
//   copies   each band's rows into the neighbour's halo rows (5 fields x 4 rows per cut
//            and direction, cudaMemcpy2DAsync between the devices' memories), on the
//            receiving slab's high-priority stream, after the sending slab's band;
//   interior the other owned rows, on the slab's main stream, after its previous band.
// So the copies and the next bands run while the interior rows are computed, and the
// halo rows are never computed (they are copied).  Hazards: a band reads halo and owned
// rows its previous interior and the copies wrote; an interior reads the owned rows its
// previous band wrote, and overwrites rows that band read; a copy reads band rows that the
// sender's next band overwrites only after the receiver's band, which follows the copy
// on the receiver's stream, and after the copy back into the sender that waits for it.
// The results are bitwise those of the whole grid stepped by one task.
//
// le_step_soa's far end (the last two rows read rows ny-5 and ny-4 instead of copies of row
// ny-1) only affects the rows next to a grid's bottom: at a cut those are halo rows, and at
// the last slab's bottom the slab's rows ny-5, ny-4 are the grid's.  So SoA tasks split too
// (one step per launch, as whole SoA tasks).
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "consts.h"
#include "le2d.h"
#include "le2d_kernels.h"

namespace {

using T = real;
using le2d::FusedPlan;
using le2d::StepConsts;

constexpr int kHalo = 4;          // rows: two steps per launch, two rows per step
constexpr int kMinSlabRows = 8;   // owned rows per slab
constexpr int kMaxSlabs = 64;
constexpr unsigned long long kPairWaitNs = 1000000000ull;

struct Slab {
  int dev = 0;
  int r0 = 0, r1 = 0;  // owned global rows
  int h0 = 0, h1 = 0;  // halo rows above / below
  int nyl = 0;         // rows of the device grid
  long long plane = 0;
  T* mem = nullptr;
  T* buf[2] = {nullptr, nullptr};
  int* d_status = nullptr;
  cudaStream_t stream = nullptr;   // interior rows
  cudaStream_t bstream = nullptr;  // boundary bands and the halo copies into this slab (high priority)
  cudaEvent_t ev_band[2] = {nullptr, nullptr};  // after the band of launch k (k & 1)
  cudaEvent_t ev_int[2] = {nullptr, nullptr};   // after the interior of launch k (k & 1)
  FusedPlan plan, plan1;
};

// Variant of each launch: FP32 two steps on warp pairs (one-step variant 2 for odd
// remainders and SoA), FP64 one step (variant 15), as for whole tasks.
int two_step_variant() { return sizeof(T) == 4 ? 13 : 15; }
int one_step_variant() { return sizeof(T) == 4 ? 2 : 15; }

}  // namespace

struct le2d_slabs {
  int nx = 0, ny = 0, stype = ST_AOS;
  long long pitch = 0;
  StepConsts<T> c;
  std::vector<Slab> s;
  int cur = 0;  // buffer holding the state (the same on every slab)
  long long launches = 0;
  int err = LE2D_OK;

  int fail(int code, const char* what, cudaError_t e = cudaSuccess) {
    if (e != cudaSuccess)
      fprintf(stderr, "le2d: slabs: %s: %s\n", what, cudaGetErrorString(e));
    else
      fprintf(stderr, "le2d: slabs: %s: %s\n", what, le2d_strerror(code));
    if (err == LE2D_OK) err = code;
    return code;
  }
};

namespace {

// Copies fields' rows [sr, sr+rows) of slab a into rows [dr, dr+rows) of slab b (buffer `buf`)
// on slab b's stream.
cudaError_t copy_rows(le2d_slabs* S, const Slab& a, int sr, Slab& b, int dr, int rows, int buf) {
  for (int k = 0; k < 5; ++k) {
    const T* src = a.buf[buf] + k * a.plane + (long long)sr * S->pitch;
    T* dst = b.buf[buf] + k * b.plane + (long long)dr * S->pitch;
    cudaError_t e = cudaMemcpy2DAsync(dst, sizeof(T) * S->pitch, src, sizeof(T) * S->pitch,
                                      sizeof(T) * S->nx, rows, cudaMemcpyDefault, b.bstream);
    if (e != cudaSuccess) return e;
  }
  return cudaSuccess;
}

// Halo rows of buffer `buf` from the neighbours' band rows, after launch k: each copy on the
// receiving slab's band stream, after the sending slab's band.
cudaError_t exchange(le2d_slabs* S, int buf, long long k) {
  const int n = (int)S->s.size();
  for (int i = 0; i + 1 < n; ++i) {
    Slab& a = S->s[i];
    Slab& b = S->s[i + 1];
    // b's top halo <- a's last kHalo owned rows; a's bottom halo <- b's first kHalo owned rows
    cudaSetDevice(b.dev);
    cudaError_t e = cudaStreamWaitEvent(b.bstream, a.ev_band[k & 1], 0);
    if (e == cudaSuccess) e = copy_rows(S, a, a.h0 + (a.r1 - a.r0) - kHalo, b, 0, kHalo, buf);
    if (e != cudaSuccess) return e;
    cudaSetDevice(a.dev);
    e = cudaStreamWaitEvent(a.bstream, b.ev_band[k & 1], 0);
    if (e == cudaSuccess) e = copy_rows(S, b, b.h0, a, a.h0 + (a.r1 - a.r0), kHalo, buf);
    if (e != cudaSuccess) return e;
  }
  return cudaSuccess;
}

void release(le2d_slabs* S) {
  for (Slab& sl : S->s) {
    cudaSetDevice(sl.dev);
    if (sl.stream) cudaStreamSynchronize(sl.stream);
    if (sl.bstream) cudaStreamSynchronize(sl.bstream);
    for (int k = 0; k < 2; ++k) {
      if (sl.ev_band[k]) cudaEventDestroy(sl.ev_band[k]);
      if (sl.ev_int[k]) cudaEventDestroy(sl.ev_int[k]);
    }
    if (sl.bstream) cudaStreamDestroy(sl.bstream);
    if (sl.stream) cudaStreamDestroy(sl.stream);
    if (sl.mem) cudaFree(sl.mem);
    if (sl.d_status) cudaFree(sl.d_status);
  }
  delete S;
}

int sync_all(le2d_slabs* S) {
  for (Slab& sl : S->s) {
    cudaSetDevice(sl.dev);
    cudaError_t e = cudaStreamSynchronize(sl.stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(sl.bstream);
    if (e != cudaSuccess) return S->fail(LE2D_ECUDA, "synchronize", e);
    int h = 0;
    e = cudaMemcpy(&h, sl.d_status, sizeof(int), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return S->fail(LE2D_ECUDA, "status read", e);
    if (h) {
      cudaMemset(sl.d_status, 0, sizeof(int));
      return S->fail(LE2D_ETIMEOUT, "a warp of a two-step tile gave up waiting for its partner");
    }
  }
  return LE2D_OK;
}

}  // namespace

extern "C" {

le2d_slabs* le2d_slabs_create(const le_task* task, int nslabs, const int* devices) {
  if (!task || nslabs < 1 || nslabs > kMaxSlabs || !devices) {
    fprintf(stderr, "le2d: le2d_slabs_create: %s\n", le2d_strerror(LE2D_EINVAL));
    return nullptr;
  }
  if (task->n.x < 3 || task->n.y < kMinSlabRows * nslabs ||
      (task->stype != ST_AOS && task->stype != ST_SOA)) {
    fprintf(stderr, "le2d: le2d_slabs_create: needs n.x >= 3 and n.y >= %d rows per slab\n",
            kMinSlabRows);
    return nullptr;
  }
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    fprintf(stderr, "le2d: le2d_slabs_create: no CUDA device\n");
    return nullptr;
  }
  for (int i = 0; i < nslabs; ++i)
    if (devices[i] < 0 || devices[i] >= ndev) {
      fprintf(stderr, "le2d: le2d_slabs_create: no device %d\n", devices[i]);
      return nullptr;
    }
  int prev = 0;
  cudaGetDevice(&prev);
  auto* S = new le2d_slabs();
  S->nx = task->n.x;
  S->ny = task->n.y;
  S->stype = task->stype;
  S->pitch = le2d::row_pitch_elems(S->nx);
  S->c = le2d::make_consts(task->dt, task->h, task->mat);
  S->s.resize(nslabs);
  cudaError_t e = cudaSuccess;
  for (int i = 0; i < nslabs && e == cudaSuccess; ++i) {
    Slab& sl = S->s[i];
    sl.dev = devices[i];
    sl.r0 = (int)((long long)S->ny * i / nslabs);
    sl.r1 = (int)((long long)S->ny * (i + 1) / nslabs);
    sl.h0 = i > 0 ? kHalo : 0;
    sl.h1 = i + 1 < nslabs ? kHalo : 0;
    sl.nyl = sl.h0 + (sl.r1 - sl.r0) + sl.h1;
    sl.plane = S->pitch * sl.nyl;
    e = cudaSetDevice(sl.dev);
    if (e == cudaSuccess) e = cudaMalloc(&sl.mem, sizeof(T) * 2 * 5 * (size_t)sl.plane);
    if (e == cudaSuccess) e = cudaMalloc(&sl.d_status, sizeof(int));
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&sl.stream, cudaStreamNonBlocking);
    int least = 0, greatest = 0;
    if (e == cudaSuccess) e = cudaDeviceGetStreamPriorityRange(&least, &greatest);
    if (e == cudaSuccess) e = cudaStreamCreateWithPriority(&sl.bstream, cudaStreamNonBlocking, greatest);
    for (int k = 0; k < 2 && e == cudaSuccess; ++k) {
      e = cudaEventCreateWithFlags(&sl.ev_band[k], cudaEventDisableTiming);
      if (e == cudaSuccess) e = cudaEventCreateWithFlags(&sl.ev_int[k], cudaEventDisableTiming);
    }
    if (e == cudaSuccess) e = cudaMemsetAsync(sl.mem, 0, sizeof(T) * 2 * 5 * (size_t)sl.plane, sl.stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(sl.d_status, 0, sizeof(int), sl.stream);
    if (e != cudaSuccess) break;
    sl.buf[0] = sl.mem;
    sl.buf[1] = sl.mem + 5 * sl.plane;
    const int v2 = two_step_variant(), v1 = one_step_variant();
    sl.plan = le2d::plan_fused<T>(S->nx, sl.nyl, v2, le2d::fused_resident_warps<T>(sl.dev, v2), 16);
    sl.plan1 = le2d::plan_fused<T>(S->nx, sl.nyl, v1, le2d::fused_resident_warps<T>(sl.dev, v1), 16);
    // peer access to the neighbour above (copies work without it, staged by the driver)
    if (i > 0 && S->s[i - 1].dev != sl.dev) {
      int can = 0;
      cudaDeviceCanAccessPeer(&can, sl.dev, S->s[i - 1].dev);
      if (can && cudaDeviceEnablePeerAccess(S->s[i - 1].dev, 0) != cudaSuccess) cudaGetLastError();
      cudaSetDevice(S->s[i - 1].dev);
      cudaDeviceCanAccessPeer(&can, S->s[i - 1].dev, sl.dev);
      if (can && cudaDeviceEnablePeerAccess(sl.dev, 0) != cudaSuccess) cudaGetLastError();
    }
  }
  cudaSetDevice(prev);
  if (e != cudaSuccess) {
    fprintf(stderr, "le2d: le2d_slabs_create: %s\n", cudaGetErrorString(e));
    release(S);
    return nullptr;
  }
  return S;
}

void le2d_slabs_destroy(le2d_slabs* S) {
  if (!S) return;
  int prev = 0;
  cudaGetDevice(&prev);
  release(S);
  cudaSetDevice(prev);
}

int le2d_slabs_rows(const le2d_slabs* S, int slab, int* r0, int* r1, int* device) {
  if (!S || slab < 0 || slab >= (int)S->s.size()) return LE2D_EINVAL;
  if (r0) *r0 = S->s[slab].r0;
  if (r1) *r1 = S->s[slab].r1;
  if (device) *device = S->s[slab].dev;
  return LE2D_OK;
}

// Each slab receives the rows [r0 - h0, r1 + h1) of the caller's grid (task layout).
int le2d_slabs_upload(le2d_slabs* S, const real* src) {
  if (!S || !src) return LE2D_EINVAL;
  int prev = 0;
  cudaGetDevice(&prev);
  const int aos = S->stype == ST_AOS;
  const long long n = (long long)S->nx * S->ny;
  int rc = LE2D_OK;
  for (Slab& sl : S->s) {
    cudaSetDevice(sl.dev);
    T* stage = sl.buf[S->cur ^ 1];
    const int g0 = sl.r0 - sl.h0;
    const size_t rows_elems = (size_t)S->nx * sl.nyl;
    cudaError_t e = cudaSuccess;
    if (aos) {
      e = cudaMemcpyAsync(stage, src + (size_t)g0 * S->nx * 5, sizeof(T) * 5 * rows_elems,
                          cudaMemcpyHostToDevice, sl.stream);
    } else {
      for (int k = 0; k < 5 && e == cudaSuccess; ++k)
        e = cudaMemcpyAsync(stage + k * rows_elems, src + k * n + (size_t)g0 * S->nx,
                            sizeof(T) * rows_elems, cudaMemcpyHostToDevice, sl.stream);
    }
    if (e == cudaSuccess)
      e = le2d::launch_pack<T>(stage, sl.buf[S->cur], S->nx, sl.nyl, S->pitch, sl.plane, aos, sl.stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(sl.stream);  // src may be pageable
    if (e != cudaSuccess) {
      rc = S->fail(LE2D_ECUDA, "upload", e);
      break;
    }
  }
  cudaSetDevice(prev);
  return rc;
}

// The owned rows of every slab into the caller's grid (task layout); synchronises.
int le2d_slabs_download(le2d_slabs* S, real* dst) {
  if (!S || !dst) return LE2D_EINVAL;
  int prev = 0;
  cudaGetDevice(&prev);
  int rc = sync_all(S);
  const int aos = S->stype == ST_AOS;
  const long long n = (long long)S->nx * S->ny;
  for (size_t i = 0; i < S->s.size() && rc == LE2D_OK; ++i) {
    Slab& sl = S->s[i];
    cudaSetDevice(sl.dev);
    T* stage = sl.buf[S->cur ^ 1];
    const int own = sl.r1 - sl.r0;
    const size_t rows_elems = (size_t)S->nx * own;
    cudaError_t e = le2d::launch_unpack<T>(sl.buf[S->cur] + (long long)sl.h0 * S->pitch, stage, S->nx,
                                           own, S->pitch, sl.plane, aos, sl.stream);
    if (aos) {
      if (e == cudaSuccess)
        e = cudaMemcpyAsync(dst + (size_t)sl.r0 * S->nx * 5, stage, sizeof(T) * 5 * rows_elems,
                            cudaMemcpyDeviceToHost, sl.stream);
    } else {
      for (int k = 0; k < 5 && e == cudaSuccess; ++k)
        e = cudaMemcpyAsync(dst + k * n + (size_t)sl.r0 * S->nx, stage + k * rows_elems,
                            sizeof(T) * rows_elems, cudaMemcpyDeviceToHost, sl.stream);
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(sl.stream);
    if (e != cudaSuccess) rc = S->fail(LE2D_ECUDA, "download", e);
  }
  cudaSetDevice(prev);
  return rc;
}

// nsteps steps: launches of two steps (one at an odd end, and for SoA grids), each a band
// and an interior launch per slab plus the halo copies.  Asynchronous: le2d_slabs_download
// (or _wait) synchronises.
int le2d_slabs_step_n(le2d_slabs* S, int nsteps) {
  if (!S || nsteps < 0) return LE2D_EINVAL;
  int prev = 0;
  cudaGetDevice(&prev);
  const int far_rot = S->stype == ST_SOA ? 1 : 0;
  const int n = (int)S->s.size();
  int rc = LE2D_OK;
  for (int left = nsteps; left > 0 && rc == LE2D_OK;) {
    const bool two = !far_rot && left >= 2 && S->s[0].plan.depth == 2;
    const long long k = S->launches;
    for (int i = 0; i < n && rc == LE2D_OK; ++i) {
      Slab& sl = S->s[i];
      cudaSetDevice(sl.dev);
      const FusedPlan& pl = two ? sl.plan : sl.plan1;
      le2d::PairCtl pc;
      pc.status = sl.d_status;
      pc.wait_ns = kPairWaitNs;
      const int own0 = sl.h0, own1 = sl.h0 + (sl.r1 - sl.r0);
      const int in0 = own0 + (i > 0 ? kHalo : 0), in1 = own1 - (i + 1 < n ? kHalo : 0);
      const T* src = sl.buf[S->cur];
      T* dst = sl.buf[S->cur ^ 1];
      // interior rows, after this slab's previous band
      cudaError_t e = cudaStreamWaitEvent(sl.stream, sl.ev_band[(k + 1) & 1], 0);
      if (e == cudaSuccess)
        e = le2d::launch_fused_rows<T>(src, dst, S->nx, sl.nyl, S->pitch, sl.plane, S->c, far_rot, pl, pc,
                                       pl.seg_len, 1, &in0, &in1, sl.stream);
      if (e == cudaSuccess) e = cudaEventRecord(sl.ev_int[k & 1], sl.stream);
      // bands beside the cuts, after this slab's previous interior (and, on this stream, the
      // halo copies into it)
      int lo[2], hi[2], nr = 0;
      if (i > 0) {
        lo[nr] = own0;
        hi[nr++] = own0 + kHalo;
      }
      if (i + 1 < n) {
        lo[nr] = own1 - kHalo;
        hi[nr++] = own1;
      }
      if (e == cudaSuccess) e = cudaStreamWaitEvent(sl.bstream, sl.ev_int[(k + 1) & 1], 0);
      if (e == cudaSuccess && nr > 0)
        e = le2d::launch_fused_rows<T>(src, dst, S->nx, sl.nyl, S->pitch, sl.plane, S->c, far_rot, pl, pc,
                                       kHalo, nr, lo, hi, sl.bstream);
      if (e == cudaSuccess) e = cudaEventRecord(sl.ev_band[k & 1], sl.bstream);
      if (e != cudaSuccess) rc = S->fail(LE2D_ECUDA, "step kernel launch", e);
    }
    if (rc) break;
    S->cur ^= 1;
    const cudaError_t e = exchange(S, S->cur, k);
    if (e != cudaSuccess) rc = S->fail(LE2D_ECUDA, "halo exchange", e);
    ++S->launches;
    left -= two ? 2 : 1;
  }
  cudaSetDevice(prev);
  return rc;
}

int le2d_slabs_wait(le2d_slabs* S) {
  if (!S) return LE2D_EINVAL;
  int prev = 0;
  cudaGetDevice(&prev);
  const int rc = sync_all(S);
  cudaSetDevice(prev);
  return rc;
}

}  // extern "C"
