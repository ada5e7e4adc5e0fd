// One grid split into row slabs over several devices (the reference's multi-GPU scheme,
// le2d cuda5/cuda6: le_core.cu:374-509, one process driving every device with peer
// copies of the rows next to each cut).
//
// Slab s owns the global rows [r0, r1) and keeps a copy of kHalo rows on each side that
// has a neighbour (none at the grid's top and bottom), so its device grid is the rows
// [r0 - h0, r1 + h1).  Every launch advances each slab with the unmodified fused kernel on
// its own grid: at a cut that grid's clamped end is wrong, but the error enters two rows per
// step, so after a launch of up to two steps the halo rows are spoiled and the owned rows
// are exact.  The halo rows are then refreshed from the neighbours' owned rows (5 fields x
// kHalo rows each way per cut, cudaMemcpy2DAsync between the devices' memories).  The
// results are therefore bitwise those of the whole grid stepped by one task.
//
// Ordering.  Each slab has a stream on its device.  A launch of slab s is queued after its
// own halo copies (same stream); a halo copy into slab s waits (event) for the launch of the
// neighbour it reads from.  The neighbour's next launch, which overwrites the other buffer,
// is queued after its own copies, which wait for slab s's launch; so no copy reads a buffer
// that is being written and no launch overwrites rows a copy has not read yet.
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
  cudaStream_t stream = nullptr;
  cudaEvent_t ev = nullptr;  // after this slab's last launch
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
                                      sizeof(T) * S->nx, rows, cudaMemcpyDefault, b.stream);
    if (e != cudaSuccess) return e;
  }
  return cudaSuccess;
}

// Refreshes every slab's halo rows (buffer `buf`) from its neighbours' owned rows.
cudaError_t exchange(le2d_slabs* S, int buf) {
  const int n = (int)S->s.size();
  for (int i = 0; i + 1 < n; ++i) {
    Slab& a = S->s[i];
    Slab& b = S->s[i + 1];
    // b's top halo <- a's last kHalo owned rows; a's bottom halo <- b's first kHalo owned rows
    cudaSetDevice(b.dev);
    cudaError_t e = cudaStreamWaitEvent(b.stream, a.ev, 0);
    if (e == cudaSuccess) e = copy_rows(S, a, a.h0 + (a.r1 - a.r0) - kHalo, b, 0, kHalo, buf);
    if (e != cudaSuccess) return e;
    cudaSetDevice(a.dev);
    e = cudaStreamWaitEvent(a.stream, b.ev, 0);
    if (e == cudaSuccess) e = copy_rows(S, b, b.h0, a, a.h0 + (a.r1 - a.r0), kHalo, buf);
    if (e != cudaSuccess) return e;
  }
  return cudaSuccess;
}

void release(le2d_slabs* S) {
  for (Slab& sl : S->s) {
    cudaSetDevice(sl.dev);
    if (sl.stream) cudaStreamSynchronize(sl.stream);
    if (sl.ev) cudaEventDestroy(sl.ev);
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
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&sl.ev, cudaEventDisableTiming);
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

// nsteps steps: launches of two steps (one at an odd end, and for SoA grids), each followed
// by the halo exchange.  Asynchronous: le2d_slabs_download (or _wait) synchronises.
int le2d_slabs_step_n(le2d_slabs* S, int nsteps) {
  if (!S || nsteps < 0) return LE2D_EINVAL;
  int prev = 0;
  cudaGetDevice(&prev);
  const int far_rot = S->stype == ST_SOA ? 1 : 0;
  int rc = LE2D_OK;
  for (int left = nsteps; left > 0 && rc == LE2D_OK;) {
    const bool two = !far_rot && left >= 2 && S->s[0].plan.depth == 2;
    for (Slab& sl : S->s) {
      cudaSetDevice(sl.dev);
      const FusedPlan& pl = two ? sl.plan : sl.plan1;
      le2d::PairCtl pc;
      pc.status = sl.d_status;
      pc.wait_ns = kPairWaitNs;
      cudaError_t e = le2d::launch_fused_step<T>(sl.buf[S->cur], sl.buf[S->cur ^ 1], S->nx, sl.nyl,
                                                 S->pitch, sl.plane, S->c, far_rot, pl, pc, sl.stream);
      if (e == cudaSuccess) e = cudaEventRecord(sl.ev, sl.stream);
      if (e != cudaSuccess) {
        rc = S->fail(LE2D_ECUDA, "step kernel launch", e);
        break;
      }
    }
    if (rc) break;
    S->cur ^= 1;
    const cudaError_t e = exchange(S, S->cur);
    if (e != cudaSuccess) rc = S->fail(LE2D_ECUDA, "halo exchange", e);
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
