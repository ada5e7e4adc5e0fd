// The le2d task API (include/le_core.h) and its extensions (include/le2d.h) on
// one B200.  Compiled once per precision: `real` is float, or double with
// -DUSE_DOUBLE (lible2d_f.so / lible2d_d.so), as the reference builds its
// simple/ solver twice (simple/Makefile:6-7).
//
// State.  The reference keeps the grid in task->grid and steps it in place
// (simple/le_core.c:605-620).  Here every task also owns a device state: two
// pitched SoA buffers (ping-pong, since a step reads the old state while writing
// the new one) registered under the task's grid pointer (the le_task struct has
// no spare field and callers keep it on their stack, simple/main.c:27).  Steps
// are queued on the task's stream and the host grid is refreshed only on
// le_save_task, le2d_sync_host and le2d_download.
//
// Errors.  The reference asserts (simple/le_core.c:89, :261, :437); this library
// never aborts or exits: it prints the cause on stderr and keeps the first error
// per task (le2d_last_error).  There is no CPU fallback: without a device, steps
// fail with LE2D_ENODEV.
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <unordered_map>

#include "consts.h"
#include "le2d.h"
#include "le2d_kernels.h"

namespace {

using T = real;
using le2d::FusedPlan;
using le2d::StepConsts;
using le2d::Sweep;

constexpr int kMinSeg = 16;  // shortest row segment of the fused kernel

struct DevTask {
  int nx = 0, ny = 0;
  long long pitch = 0, plane = 0;
  T* mem = nullptr;
  T* buf[2] = {nullptr, nullptr};
  int cur = 0;
  double* d_diag = nullptr;
  int* d_status = nullptr;    // set by a warp-pair launch whose wait gave up
  bool pairs_queued = false;  // warp-pair launches since d_status was last read
  int stall_pair = -1;        // test hook (LE2D_TEST_STALL_PAIR): tile whose producer stalls
  cudaStream_t stream = nullptr;
  cudaEvent_t ev[2] = {nullptr, nullptr};
  bool pinned = false;     // task->grid from cudaHostAlloc
  bool host_newer = false; // task->grid holds a newer state than the device
  bool dev_newer = false;  // the device holds a newer state than task->grid
  bool has_device = false;
  int err = LE2D_OK;
  int method = LE2D_METHOD_FUSED;
  FusedPlan plan;
  FusedPlan plan1;  // depth-1 plan for single steps when `plan` has depth 2
  // One le_step call held back under a two-step plan, so that the next call makes a
  // two-step launch with it; queued by itself before anything else touches the state.
  bool pending = false;
  StepConsts<T> pending_c;
  long long steps = 0;
  double sim_time = 0.0;
  // CUDA graph of kGraphSteps steps starting from buffer graph_cur.
  cudaGraphExec_t graph = nullptr;
  int graph_cur = -1, graph_method = -1, graph_far_rot = -1;
  bool graph_halves = false;
  StepConsts<T> graph_consts;
  // Fused launches in halves (halves_launch): hs[0] the band of rows around the middle of
  // the grid (high priority), hs[1] / hs[2] the rows above / below it; hev[i][k & 1] after
  // stream i's part of launch k of the current sequence, hk launches so far.
  bool halves = false;
  cudaStream_t hs[3] = {nullptr, nullptr, nullptr};
  cudaEvent_t hev[3][2] = {{nullptr, nullptr}, {nullptr, nullptr}, {nullptr, nullptr}};
  cudaEvent_t fork_ev = nullptr;
  long long hk = 0;
};

constexpr int kGraphSteps = 64;  // even, so a replay leaves the current buffer unchanged
// Bound of every wait between the two warps of a warp-pair tile (they share a block, so a
// wait that long means a fault in the kernel, not a slow partner).
constexpr unsigned long long kPairWaitNs = 1000000000ull;

// Fused launches in halves.  One launch over the whole grid ends on a partly idle device:
// its last wave of tiles thins out before the next launch, which depends on all of it,
// starts.  Cut in three -- the band of kBand rows on each side of the middle row, the rows
// above it and the rows below it -- a launch's parts depend on the previous launch's only
// where their stencils meet: each interior part on the previous band (which it reads, and
// whose reads of its rows it must not overtake), the band on both previous interior parts.
// So the upper and lower parts run on streams of their own and overlap each other's ends,
// as the row slabs of two devices do (slabs.cu), without copies: the parts share the
// task's buffers and write disjoint rows.  The stencil of a launch reaches 4 rows (two
// steps of two), so kBand = 4.  Bitwise the same results as whole launches.
constexpr int kBand = 4;
constexpr int kMinHalvesRows = 256;  // grids with fewer rows launch whole

// Whether a task's fused launches go in halves: on grids of at least kMinHalvesRows rows.
// Measured (Gnu/s, best whole launch / halves, each at its fitted segment length): FP32
// 1024^2 47.3 / 50.9, 3000^2 159.0 / 161.3, 4096^2 158.5 / 176.2, 6000^2 176.5 / 191.8,
// 8192^2 181.8 / 195.2, 16384^2 192.7 / 197.2, 8192 x 2048 158.7 / 179.5, 2048 x 8192 158.3 /
// 167.7, 2048^2 131.1 / 128.7; FP64 (whole segment lengths) 2048^2 44.6 / 46.1, 4096^2 51.1 /
// 53.7, 8192^2 55.9 / 57.2.  LE2D_HALVES=1 / 0 overrides it (on every grid of at least
// 4 kBand rows / never).
bool halves_for(int ny) {
  static const int mode = [] {  // read once, thread-safely
    const char* e = getenv("LE2D_HALVES");
    return e ? (atoi(e) != 0 ? 1 : 0) : -1;
  }();
  if (mode == 0 || ny < 4 * kBand) return false;
  return mode == 1 || ny >= kMinHalvesRows;
}

cudaError_t create_halves(DevTask* d) {
  int lo = 0, hi = 0;
  cudaError_t e = cudaDeviceGetStreamPriorityRange(&lo, &hi);
  if (e == cudaSuccess) e = cudaStreamCreateWithPriority(&d->hs[0], cudaStreamNonBlocking, hi);
  for (int i = 1; i < 3 && e == cudaSuccess; ++i) e = cudaStreamCreateWithFlags(&d->hs[i], cudaStreamNonBlocking);
  for (int i = 0; i < 3 && e == cudaSuccess; ++i)
    for (int j = 0; j < 2 && e == cudaSuccess; ++j) e = cudaEventCreateWithFlags(&d->hev[i][j], cudaEventDisableTiming);
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&d->fork_ev, cudaEventDisableTiming);
  return e;
}

void destroy_halves(DevTask* d) {
  for (int i = 0; i < 3; ++i) {
    if (d->hs[i]) {
      cudaStreamSynchronize(d->hs[i]);
      cudaStreamDestroy(d->hs[i]);
    }
    for (int j = 0; j < 2; ++j)
      if (d->hev[i][j]) cudaEventDestroy(d->hev[i][j]);
  }
  if (d->fork_ev) cudaEventDestroy(d->fork_ev);
}

// Starts a sequence of launches in halves: the three streams wait for the task's stream.
cudaError_t halves_begin(DevTask* d) {
  d->hk = 0;
  cudaError_t e = cudaEventRecord(d->fork_ev, d->stream);
  for (int i = 0; i < 3 && e == cudaSuccess; ++i) e = cudaStreamWaitEvent(d->hs[i], d->fork_ev, 0);
  return e;
}

// Ends it: the task's stream waits for the three streams.
cudaError_t halves_end(DevTask* d) {
  cudaError_t e = cudaSuccess;
  for (int i = 0; i < 3 && e == cudaSuccess; ++i) {
    cudaEvent_t ev = d->hev[i][d->hk & 1];
    e = cudaEventRecord(ev, d->hs[i]);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(d->stream, ev, 0);
  }
  return e;
}

// Launch k of the sequence, from a into b, in three parts.
cudaError_t halves_launch(DevTask* d, const T* a, T* b, const StepConsts<T>& c, const FusedPlan& pl,
                          const le2d::PairCtl& pc) {
  const long long k = d->hk;
  const int mid = d->ny / 2;
  const int lo[3] = {mid - kBand, 0, mid + kBand}, hi[3] = {mid + kBand, mid - kBand, d->ny};
  cudaError_t e = cudaSuccess;
  if (k > 0) {  // the band after both interior parts of launch k-1
    e = cudaStreamWaitEvent(d->hs[0], d->hev[1][(k + 1) & 1], 0);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(d->hs[0], d->hev[2][(k + 1) & 1], 0);
  }
  if (e == cudaSuccess)
    e = le2d::launch_fused_rows<T>(a, b, d->nx, d->ny, d->pitch, d->plane, c, 0, pl, pc, 2 * kBand, 1, &lo[0],
                                   &hi[0], d->hs[0]);
  if (e == cudaSuccess) e = cudaEventRecord(d->hev[0][k & 1], d->hs[0]);
  for (int i = 1; i < 3 && e == cudaSuccess; ++i) {  // each interior part after the band of launch k-1
    if (k > 0) e = cudaStreamWaitEvent(d->hs[i], d->hev[0][(k + 1) & 1], 0);
    if (e == cudaSuccess)
      e = le2d::launch_fused_rows<T>(a, b, d->nx, d->ny, d->pitch, d->plane, c, 0, pl, pc, pl.seg_len, 1, &lo[i],
                                     &hi[i], d->hs[i]);
    if (e == cudaSuccess) e = cudaEventRecord(d->hev[i][k & 1], d->hs[i]);
  }
  ++d->hk;
  return e;
}

std::mutex g_mu;
std::unordered_map<const void*, DevTask*> g_tasks;

int device_count() {
  static const int n = [] {  // queried once, thread-safely
    int c = 0;
    const int k = cudaGetDeviceCount(&c) == cudaSuccess ? c : 0;
    if (k == 0) cudaGetLastError();
    return k;
  }();
  return n;
}

int record(DevTask* d, int code, const char* what, cudaError_t e = cudaSuccess) {
  if (e != cudaSuccess)
    fprintf(stderr, "le2d: %s: %s\n", what, cudaGetErrorString(e));
  else
    fprintf(stderr, "le2d: %s: %s\n", what, le2d_strerror(code));
  if (d && d->err == LE2D_OK) d->err = code;
  return code;
}

DevTask* lookup(const le_task* task) {
  if (!task || !task->grid) return nullptr;
  std::lock_guard<std::mutex> lk(g_mu);
  auto it = g_tasks.find(task->grid);
  return it == g_tasks.end() ? nullptr : it->second;
}

long long row_pitch(int nx) { return le2d::row_pitch_elems(nx); }

// Fused-kernel variant used for new tasks: LE2D_FUSED_VARIANT if set, else the fastest
// measured on large grids (FP32: two steps per launch on producer / consumer warp pairs,
// 4 columns per lane, 16 warps per SM, one pair per block, boundary tiles first, interior
// tiles on the lean loops; FP64: one step per launch, 2 columns per lane, boundary tiles
// first, interior tiles on the lean one-step loop in 128 registers, 16 warps per SM -- the
// FP64 two-step variants measured slower).
int default_variant() {
  static const int v = [] {  // read once, thread-safely
    const int dflt = sizeof(T) == 4 ? 13 : 15;
    const char* e = getenv("LE2D_FUSED_VARIANT");
    const int x = e ? atoi(e) : dflt;
    return x < 0 || x >= le2d::fused_variant_count<T>() ? dflt : x;
  }();
  return v;
}

// Work decomposition of the fused kernel for this task; seg_len 0 = fill the device once.
void replan(DevTask* d, int variant, int seg_len) {
  int dev = 0;
  cudaGetDevice(&dev);
  const int resident = le2d::fused_resident_warps<T>(dev, variant);
  d->halves = d->hs[0] != nullptr && halves_for(d->ny);
  le2d::FusedPlan p = le2d::plan_fused<T>(d->nx, d->ny, variant, resident, kMinSeg, d->halves);
  if (seg_len > 0) {  // explicit segment length (tuning)
    const int wpb = p.threads / 32 / p.warps_per_task;  // tiles per block
    p.seg_len = seg_len < d->ny ? seg_len : d->ny;
    p.nsegs = (d->ny + p.seg_len - 1) / p.seg_len;
    p.ntasks = p.nstrips * p.nsegs;
    p.blocks = (p.ntasks + wpb - 1) / wpb;
  }
  d->plan = p;
  d->plan1 = p;
  if (p.depth != 1) {  // odd remainders and le_step_soa run single steps
    const int v = sizeof(T) == 4 ? 2 : 15;  // the fastest one-step variant
    d->plan1 = le2d::plan_fused<T>(d->nx, d->ny, v, le2d::fused_resident_warps<T>(dev, v), kMinSeg);
  }
  if (d->graph) cudaGraphExecDestroy(d->graph);
  d->graph = nullptr;
}

// Step constants from the task as it is now (the caller may change dt between steps).
StepConsts<T> make_consts(const le_task* t) { return le2d::make_consts(t->dt, t->h, t->mat); }

// ---- autotuner: fastest fused-kernel plan per size class ----

struct Tuned {
  int variant = 0, seg_len = 0;
  double nu_s = 0.0;
};
std::mutex g_tune_mu;
std::map<std::pair<int, int>, Tuned> g_tuned;

int ceil_log2(int n) {
  int k = 0;
  while ((1 << k) < n) ++k;
  return k;
}
std::pair<int, int> size_class(int nx, int ny) { return {ceil_log2(nx), ceil_log2(ny)}; }

void release(DevTask* d);
cudaError_t queue_step(DevTask* d, const StepConsts<T>& c, int far_rot, int method, int* cur,
                       int max_steps, int* done, bool halves = false);

// Times every variant x segment length on a scratch nx x ny state (a disk of radius
// min(nx,ny)/4 on a zero field, c1 = 2, c2 = 1, rho = 1, Courant number 0.5).
int tune_size(int nx, int ny, Tuned* best) {
  DevTask* d = new DevTask();
  d->nx = nx;
  d->ny = ny;
  d->pitch = row_pitch(nx);
  d->plane = d->pitch * ny;
  d->has_device = true;
  cudaError_t e = cudaMalloc(&d->mem, sizeof(T) * 2 * 5 * (size_t)d->plane);
  if (e != cudaSuccess) {
    cudaGetLastError();
    d->mem = nullptr;
    release(d);
    return LE2D_ENOMEM;
  }
  d->buf[0] = d->mem;
  d->buf[1] = d->mem + 5 * d->plane;
  e = cudaStreamCreateWithFlags(&d->stream, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaEventCreate(&d->ev[0]);
  if (e == cudaSuccess) e = cudaEventCreate(&d->ev[1]);
  if (e == cudaSuccess) e = cudaMalloc(&d->d_status, sizeof(int));
  if (e == cudaSuccess) e = cudaMemsetAsync(d->d_status, 0, sizeof(int), d->stream);
  if (e == cudaSuccess) e = cudaMemsetAsync(d->mem, 0, sizeof(T) * 2 * 5 * (size_t)d->plane, d->stream);
  if (e == cudaSuccess)
    e = le2d::launch_set_ball<T>(d->buf[0], nx, ny, d->pitch, d->plane, 1, 1, nx / 2, ny / 2,
                                 (nx < ny ? nx : ny) / 4, 1, d->stream);
  le_material m;
  le_init_material(2, 1, 1, &m);
  le_vec2 h;
  h.x = h.y = 1;
  const StepConsts<T> c = le2d::make_consts((real)0.25, h, m);
  const int segs[] = {0, 16, 24, 32, 48, 64, 96, 128, 192, 256};
  best->nu_s = -1.0;
  for (int v = 0; v < le2d::fused_variant_count<T>() && e == cudaSuccess; ++v) {
    for (int s : segs) {
      if (s > ny) continue;
      replan(d, v, s);
      float ms = 0.0f;
      int steps = 0;
      for (int k = 0; k < 2 && e == cudaSuccess; ++k)
        e = queue_step(d, c, 0, LE2D_METHOD_FUSED, &d->cur, 2, &steps);
      // estimate one launch, then time enough launches for ~3 ms
      if (e == cudaSuccess) e = cudaEventRecord(d->ev[0], d->stream);
      for (int k = 0; k < 3 && e == cudaSuccess; ++k)
        e = queue_step(d, c, 0, LE2D_METHOD_FUSED, &d->cur, 2, &steps);
      if (e == cudaSuccess) e = cudaEventRecord(d->ev[1], d->stream);
      if (e == cudaSuccess) e = cudaEventSynchronize(d->ev[1]);
      if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, d->ev[0], d->ev[1]);
      if (e != cudaSuccess) break;
      int reps = (int)(3.0f / (ms / 3.0f + 1e-4f));
      reps = reps < 5 ? 5 : (reps > 400 ? 400 : reps);
      steps = 0;
      e = cudaEventRecord(d->ev[0], d->stream);
      for (int k = 0; k < reps && e == cudaSuccess; ++k)
        e = queue_step(d, c, 0, LE2D_METHOD_FUSED, &d->cur, 2, &steps);
      if (e == cudaSuccess) e = cudaEventRecord(d->ev[1], d->stream);
      if (e == cudaSuccess) e = cudaEventSynchronize(d->ev[1]);
      if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, d->ev[0], d->ev[1]);
      if (e != cudaSuccess) break;
      const double nus = (double)nx * ny * steps / (ms * 1e-3);
      if (nus > best->nu_s) {
        best->nu_s = nus;
        best->variant = v;
        best->seg_len = s;
      }
    }
  }
  release(d);
  if (e != cudaSuccess) {
    fprintf(stderr, "le2d: autotune: %s\n", cudaGetErrorString(e));
    return LE2D_ECUDA;
  }
  return LE2D_OK;
}

// The tuned plan of a task's size class, tuning it first under LE2D_AUTOTUNE=1.
bool tuned_plan(int nx, int ny, Tuned* t) {
  if (getenv("LE2D_FUSED_VARIANT")) return false;  // an explicit variant wins
  const auto key = size_class(nx, ny);
  {
    std::lock_guard<std::mutex> lk(g_tune_mu);
    auto it = g_tuned.find(key);
    if (it != g_tuned.end()) {
      *t = it->second;
      return true;
    }
  }
  const char* a = getenv("LE2D_AUTOTUNE");
  if (!a || atoi(a) == 0) return false;
  if (tune_size(nx, ny, t) != LE2D_OK) return false;
  std::lock_guard<std::mutex> lk(g_tune_mu);
  g_tuned[key] = *t;
  return true;
}

bool same_consts(const StepConsts<T>& a, const StepConsts<T>& b) {
  return memcmp(&a, &b, sizeof(a)) == 0;
}

// After the task's stream has drained: reports (once) a warp-pair launch whose wait gave up.
int check_pairs(DevTask* d) {
  if (!d->pairs_queued || !d->d_status) return LE2D_OK;
  d->pairs_queued = false;
  int h = 0;
  cudaError_t e = cudaMemcpy(&h, d->d_status, sizeof(int), cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) return record(d, LE2D_ECUDA, "status read", e);
  if (h == 0) return LE2D_OK;
  cudaMemset(d->d_status, 0, sizeof(int));
  return record(d, LE2D_ETIMEOUT, "step: a warp of a two-step tile gave up waiting for its partner");
}

int upload_raw(DevTask* d, const T* host, int aos) {
  const size_t bytes = sizeof(T) * 5 * (size_t)d->nx * d->ny;
  T* stage = d->buf[d->cur ^ 1];
  cudaError_t e = cudaMemcpyAsync(stage, host, bytes, cudaMemcpyHostToDevice, d->stream);
  if (e != cudaSuccess) return record(d, LE2D_ECUDA, "upload", e);
  e = le2d::launch_pack<T>(stage, d->buf[d->cur], d->nx, d->ny, d->pitch, d->plane, aos, d->stream);
  if (e != cudaSuccess) return record(d, LE2D_ECUDA, "pack kernel", e);
  return LE2D_OK;
}

int download_raw(DevTask* d, T* host, int aos) {
  const size_t bytes = sizeof(T) * 5 * (size_t)d->nx * d->ny;
  T* stage = d->buf[d->cur ^ 1];
  cudaError_t e =
      le2d::launch_unpack<T>(d->buf[d->cur], stage, d->nx, d->ny, d->pitch, d->plane, aos, d->stream);
  if (e != cudaSuccess) return record(d, LE2D_ECUDA, "unpack kernel", e);
  e = cudaMemcpyAsync(host, stage, bytes, cudaMemcpyDeviceToHost, d->stream);
  if (e != cudaSuccess) return record(d, LE2D_ECUDA, "download", e);
  e = cudaStreamSynchronize(d->stream);
  if (e != cudaSuccess) return record(d, LE2D_ECUDA, "download sync", e);
  return check_pairs(d);
}

int ensure_device_current(DevTask* d, le_task* task) {
  if (!d->has_device) return record(d, LE2D_ENODEV, "no CUDA device");
  if (d->host_newer) {
    const int rc = upload_raw(d, task->grid, task->stype == ST_AOS);
    if (rc) return rc;
    d->host_newer = false;
  }
  return LE2D_OK;
}

int ensure_host_current(DevTask* d, le_task* task) {
  if (d->dev_newer) {
    const int rc = download_raw(d, task->grid, task->stype == ST_AOS);
    if (rc) return rc;
    d->dev_newer = false;
  }
  return LE2D_OK;
}

// Queues one launch of at most max_steps (>= 1) steps from buf[cur] and adds the steps it
// makes to *done (halves: a fused launch on clamped ends goes in halves, inside a sequence
// that halves_begin opened).  The fused kernel writes buf[cur^1] and flips cur -- two steps when the
// plan has temporal-block depth 2 and two are wanted (clamped ends only), else one; the
// split scheme sweeps x into buf[cur^1] and y back into buf[cur].
cudaError_t queue_step(DevTask* d, const StepConsts<T>& c, int far_rot, int method, int* cur,
                       int max_steps, int* done, bool halves) {
  T* a = d->buf[*cur];
  T* b = d->buf[*cur ^ 1];
  if (method == LE2D_METHOD_SPLIT) {
    cudaError_t e = le2d::launch_split_sweep<T>(0, a, b, d->nx, d->ny, d->pitch, d->plane, c.x,
                                                c.x.k1, c.x.k2, 0, d->stream);
    if (e != cudaSuccess) return e;
    *done += 1;
    return le2d::launch_split_sweep<T>(1, b, a, d->nx, d->ny, d->pitch, d->plane, c.y, c.y.k1,
                                       c.y.k2, far_rot, d->stream);
  }
  const bool two = d->plan.depth == 2 && max_steps >= 2 && !far_rot;
  const FusedPlan& pl = two ? d->plan : d->plan1;
  if (pl.warps_per_task == 2) d->pairs_queued = true;
  le2d::PairCtl pc;
  pc.status = d->d_status;
  pc.wait_ns = kPairWaitNs;
  pc.stall_task = d->stall_pair;
  cudaError_t e = halves && !far_rot
                      ? halves_launch(d, a, b, c, pl, pc)
                      : le2d::launch_fused_step<T>(a, b, d->nx, d->ny, d->pitch, d->plane, c, far_rot, pl, pc,
                                                   d->stream);
  *cur ^= 1;
  *done += pl.depth;
  return e;
}

// Queues a held-back le_step (one step) before the state is used otherwise.
int flush_pending(DevTask* d) {
  if (!d->pending) return LE2D_OK;
  d->pending = false;
  int done = 0;
  const cudaError_t e = queue_step(d, d->pending_c, 0, d->method, &d->cur, 1, &done);
  return e == cudaSuccess ? LE2D_OK : record(d, LE2D_ECUDA, "step kernel launch", e);
}

// lookup() for entry points that read, write or wait for the device state.
DevTask* lookup_sync(const le_task* task) {
  DevTask* d = lookup(task);
  if (d) flush_pending(d);
  return d;
}

int run_steps(le_task* task, int nsteps, bool soa_entry, float* ms) {
  DevTask* d = lookup(task);
  if (!d) {
    fprintf(stderr, "le2d: step: task was not created by le_init_task\n");
    return LE2D_ENOTASK;
  }
  if (nsteps < 0) return record(d, LE2D_EINVAL, "step count < 0");
  if (soa_entry ? task->stype != ST_SOA : task->stype != ST_AOS)
    return record(d, LE2D_ESTYPE, soa_entry ? "le_step_soa needs an ST_SOA task"
                                            : "le_step needs an ST_AOS task");
  if (d->nx < 3 || d->ny < 3) return record(d, LE2D_EINVAL, "step: the scheme needs n.x, n.y >= 3");
  int rc = ensure_device_current(d, task);
  if (rc) return rc;
  const StepConsts<T> c = make_consts(task);
  const int far_rot = soa_entry ? 1 : 0;
  // One le_step call under a two-step plan: held back, and launched as two steps together
  // with the next call (same constants); any other use of the state queues it first.
  if (nsteps == 1 && !soa_entry && !ms && d->method == LE2D_METHOD_FUSED && d->plan.depth == 2) {
    if (d->pending && same_consts(d->pending_c, c)) {
      d->pending = false;
      int done = 0;
      const cudaError_t e1 = queue_step(d, c, 0, d->method, &d->cur, 2, &done);
      if (e1 != cudaSuccess) return record(d, LE2D_ECUDA, "step kernel launch", e1);
    } else {
      rc = flush_pending(d);
      if (rc) return rc;
      d->pending = true;
      d->pending_c = c;
    }
    d->sim_time += (double)task->dt;
    d->steps += 1;
    d->dev_newer = true;
    return LE2D_OK;
  }
  rc = flush_pending(d);
  if (rc) return rc;
  cudaError_t e = cudaSuccess;
  if (ms) {
    e = cudaEventRecord(d->ev[0], d->stream);
    if (e != cudaSuccess) return record(d, LE2D_ECUDA, "event record", e);
  }
  int left = nsteps;
  // fused launches on clamped ends in halves (halves_launch) on grids tall enough
  const bool halves = d->halves && d->method == LE2D_METHOD_FUSED && !far_rot;
  // Long runs replay a captured graph of kGraphSteps steps (even count: buffers end where
  // they started).
  while (left >= kGraphSteps) {
    const bool valid = d->graph && d->graph_cur == d->cur && d->graph_method == d->method &&
                       d->graph_far_rot == far_rot && d->graph_halves == halves &&
                       same_consts(d->graph_consts, c);
    if (!valid) {
      if (d->graph) cudaGraphExecDestroy(d->graph);
      d->graph = nullptr;
      cudaGraph_t g = nullptr;
      e = cudaStreamBeginCapture(d->stream, cudaStreamCaptureModeThreadLocal);
      if (e != cudaSuccess) return record(d, LE2D_ECUDA, "graph capture", e);
      int cur = d->cur;
      if (halves) e = halves_begin(d);
      for (int s = 0; s < kGraphSteps && e == cudaSuccess;)
        e = queue_step(d, c, far_rot, d->method, &cur, kGraphSteps - s, &s, halves);
      if (halves && e == cudaSuccess) e = halves_end(d);
      cudaError_t e2 = cudaStreamEndCapture(d->stream, &g);
      if (e != cudaSuccess || e2 != cudaSuccess)
        return record(d, LE2D_ECUDA, "graph capture", e != cudaSuccess ? e : e2);
      e = cudaGraphInstantiate(&d->graph, g, 0);
      cudaGraphDestroy(g);
      if (e != cudaSuccess) return record(d, LE2D_ECUDA, "graph instantiate", e);
      d->graph_cur = d->cur;
      d->graph_method = d->method;
      d->graph_far_rot = far_rot;
      d->graph_halves = halves;
      d->graph_consts = c;
    }
    e = cudaGraphLaunch(d->graph, d->stream);
    if (e != cudaSuccess) return record(d, LE2D_ECUDA, "graph launch", e);
    left -= kGraphSteps;
  }
  if (left > 0 && halves) {
    e = halves_begin(d);
    if (e != cudaSuccess) return record(d, LE2D_ECUDA, "step kernel launch", e);
  }
  while (left > 0) {
    int done = 0;
    e = queue_step(d, c, far_rot, d->method, &d->cur, left, &done, halves);
    if (e != cudaSuccess) return record(d, LE2D_ECUDA, "step kernel launch", e);
    left -= done;
    if (left == 0 && halves) {
      e = halves_end(d);
      if (e != cudaSuccess) return record(d, LE2D_ECUDA, "step kernel launch", e);
    }
  }
  if (ms) {
    e = cudaEventRecord(d->ev[1], d->stream);
    if (e == cudaSuccess) e = cudaEventSynchronize(d->ev[1]);
    if (e == cudaSuccess) e = cudaEventElapsedTime(ms, d->ev[0], d->ev[1]);
    if (e != cudaSuccess) return record(d, LE2D_ECUDA, "step timing", e);
    const int rc2 = check_pairs(d);
    if (rc2) return rc2;
  }
  // FP64 simulated-time accumulator: one dt per step.
  for (int s = 0; s < nsteps; ++s) d->sim_time += (double)task->dt;
  d->steps += nsteps;
  if (nsteps > 0) d->dev_newer = true;
  return LE2D_OK;
}

void release(DevTask* d) {
  if (d->graph) cudaGraphExecDestroy(d->graph);
  destroy_halves(d);
  if (d->ev[0]) cudaEventDestroy(d->ev[0]);
  if (d->ev[1]) cudaEventDestroy(d->ev[1]);
  if (d->stream) {
    cudaStreamSynchronize(d->stream);
    cudaStreamDestroy(d->stream);
  }
  if (d->mem) cudaFree(d->mem);
  if (d->d_diag) cudaFree(d->d_diag);
  if (d->d_status) cudaFree(d->d_status);
  delete d;
}

// Host le_set_ball loop: position h*i in real, squared distance in real, sqrt and the
// test against r in double, overwrite sxx and syy (simple/le_core.c:71-94).
void set_ball_host(le_task* t, const le_vec2 c, const real r, const real s) {
  const long long plane = (long long)t->n.x * t->n.y;
  for (int i = 0; i < t->n.x; i++) {
    for (int j = 0; j < t->n.y; j++) {
      const real px = t->h.x * i;
      const real py = t->h.y * j;
      const real dx = px - c.x;
      const real dy = py - c.y;
      if (sqrt(dx * dx + dy * dy) < r) {
        const long long q = i + (long long)j * t->n.x;
        if (t->stype == ST_AOS) {
          t->grid[q * 5 + 2] = s;
          t->grid[q * 5 + 4] = s;
        } else {
          t->grid[2 * plane + q] = s;
          t->grid[4 * plane + q] = s;
        }
      }
    }
  }
}

}  // namespace

extern "C" {

const char* le2d_strerror(int code) {
  switch (code) {
    case LE2D_OK: return "ok";
    case LE2D_EINVAL: return "invalid argument";
    case LE2D_ENOTASK: return "task not created by le_init_task";
    case LE2D_ESTYPE: return "wrong storage type for this step function";
    case LE2D_ECUDA: return "CUDA error";
    case LE2D_ENOMEM: return "out of memory";
    case LE2D_ENODEV: return "no CUDA device";
    case LE2D_EBUDGET: return "exceeds the HBM budget";
    case LE2D_ETIMEOUT: return "device wait timed out";
    case LE2D_ESTATE: return "not allowed in the current state";
    default: return "unknown error";
  }
}

int le2d_set_device(int device) {
  if (device < 0 || device >= device_count()) return LE2D_ENODEV;
  cudaError_t e = cudaSetDevice(device);
  return e == cudaSuccess ? LE2D_OK : record(nullptr, LE2D_ECUDA, "le2d_set_device", e);
}

// simple/le_core.c:171-187, same expressions and type promotions.
void le_init_material(const real c1, const real c2, const real rho, le_material* m) {
  m->c1 = c1;
  m->c2 = c2;
  m->rho = rho;
  m->irhoc1 = 1.0 / (c1 * rho);
  m->irhoc2 = 1.0 / (c2 * rho);
  m->rhoc1 = c1 * rho;
  m->rhoc2 = c2 * rho;
  const real mu = rho * c2 * c2;
  const real la = rho * c1 * c1 - 2.0 * mu;
  m->rhoc3 = rho * c1 * la / (la + 2.0 * mu);
}

size_t le2d_task_device_bytes(int nx, int ny) {
  if (nx < 1 || ny < 1) return 0;
  return sizeof(T) * 2 * 5 * (size_t)row_pitch(nx) * (size_t)ny + 16 * sizeof(double);
}

void le_init_task(le_task* task, const real dt, const le_vec2 h, const le_material mat,
                  const le_point2 n, const int stype) {
  task->dt = dt;
  task->h = h;
  task->mat = mat;
  task->n = n;
  task->stype = stype;
  task->grid = nullptr;
  if (n.x < 1 || n.y < 1) {
    fprintf(stderr, "le2d: le_init_task: bad grid size %d x %d\n", n.x, n.y);
    return;
  }
  const size_t bytes = sizeof(le_node) * (size_t)n.x * n.y;
  DevTask* d = new DevTask();
  d->nx = n.x;
  d->ny = n.y;
  d->has_device = device_count() > 0;
  void* hp = nullptr;
  if (d->has_device && cudaHostAlloc(&hp, bytes, cudaHostAllocDefault) == cudaSuccess) {
    d->pinned = true;
  } else {
    if (d->has_device) cudaGetLastError();
    hp = malloc(bytes);
  }
  if (!hp) {
    fprintf(stderr, "le2d: le_init_task: host allocation of %zu bytes failed\n", bytes);
    delete d;
    return;
  }
  memset(hp, 0, bytes);
  task->grid = (real*)hp;
  if (n.x < 3 || n.y < 3) record(d, LE2D_EINVAL, "le_init_task: the scheme needs n.x, n.y >= 3");
  if (stype != ST_AOS && stype != ST_SOA) record(d, LE2D_EINVAL, "le_init_task: unknown stype");
  if (d->has_device) {
    d->pitch = row_pitch(n.x);
    d->plane = d->pitch * n.y;
    const size_t dbytes = sizeof(T) * 2 * 5 * (size_t)d->plane;
    cudaError_t e = cudaMalloc(&d->mem, dbytes);
    if (e != cudaSuccess) {
      record(d, LE2D_ENOMEM, "le_init_task: device state", e);
      d->mem = nullptr;
      d->has_device = false;
    } else {
      d->buf[0] = d->mem;
      d->buf[1] = d->mem + 5 * d->plane;
      e = cudaStreamCreateWithFlags(&d->stream, cudaStreamNonBlocking);
      if (e == cudaSuccess) e = cudaEventCreate(&d->ev[0]);
      if (e == cudaSuccess) e = cudaEventCreate(&d->ev[1]);
      if (e == cudaSuccess) e = cudaMalloc(&d->d_diag, 16 * sizeof(double));
      if (e == cudaSuccess) e = create_halves(d);
      if (e == cudaSuccess) e = cudaMalloc(&d->d_status, sizeof(int));
      if (e == cudaSuccess) e = cudaMemsetAsync(d->d_status, 0, sizeof(int), d->stream);
      if (e == cudaSuccess) e = cudaMemsetAsync(d->mem, 0, dbytes, d->stream);
      if (e != cudaSuccess) {
        record(d, LE2D_ECUDA, "le_init_task: device setup", e);
        d->has_device = false;
      }
      // Test hook for the bounded waits of warp-pair tiles: the producer of this tile
      // hands nothing over, so the step ends with a timeout status instead of results.
      if (const char* st = getenv("LE2D_TEST_STALL_PAIR")) d->stall_pair = atoi(st);
      Tuned tp;
      if (tuned_plan(n.x, n.y, &tp))
        replan(d, tp.variant, tp.seg_len);
      else
        replan(d, default_variant(), 0);
    }
  } else {
    record(d, LE2D_ENODEV, "le_init_task");
  }
  std::lock_guard<std::mutex> lk(g_mu);
  g_tasks[task->grid] = d;
}

void le_free_task(le_task* task) {
  if (!task || !task->grid) return;
  DevTask* d = nullptr;
  {
    std::lock_guard<std::mutex> lk(g_mu);
    auto it = g_tasks.find(task->grid);
    if (it != g_tasks.end()) {
      d = it->second;
      g_tasks.erase(it);
    }
  }
  const bool pinned = d && d->pinned;
  if (d) release(d);
  if (pinned)
    cudaFreeHost(task->grid);
  else
    free(task->grid);
  task->grid = nullptr;
}

void le_set_ball(le_task* t, const le_vec2 c, const real r, const real s) {
  DevTask* d = lookup_sync(t);
  if (t->stype != ST_AOS && t->stype != ST_SOA) {
    record(d, LE2D_EINVAL, "le_set_ball: unknown stype");
    return;
  }
  if (d && d->has_device && !d->host_newer) {
    cudaError_t e = le2d::launch_set_ball<T>(d->buf[d->cur], d->nx, d->ny, d->pitch, d->plane,
                                             t->h.x, t->h.y, c.x, c.y, r, s, d->stream);
    if (e != cudaSuccess) {
      record(d, LE2D_ECUDA, "le_set_ball kernel", e);
      return;
    }
    d->dev_newer = true;
    return;
  }
  if (d && d->dev_newer && ensure_host_current(d, t)) return;
  set_ball_host(t, c, r, s);
  if (d) d->host_newer = true;
}

// simple/le_core.c:130-169 with write_float :99-111: header, then |v| as big-endian float32.
// When the device holds the newest state, |v| is formed there (the same bytes, see
// launch_vtk_speed) and only those 4 bytes per node cross to the host, not the 20 of the
// full state; task->grid is then left as it is (le2d_sync_host refreshes it).
int le_save_task(le_task* t, const char* file) {
  DevTask* d = lookup_sync(t);
  const long long n = (long long)t->n.x * t->n.y;
  unsigned char* body = (unsigned char*)malloc(4 * (size_t)(n > 0 ? n : 1));
  if (!body) {
    fprintf(stderr, "le2d: le_save_task: host allocation failed\n");
    return 1;
  }
  if (d && d->has_device && !d->host_newer) {
    unsigned* scratch = reinterpret_cast<unsigned*>(d->buf[d->cur ^ 1]);  // the idle buffer
    cudaError_t e = le2d::launch_vtk_speed<T>(d->buf[d->cur], d->nx, d->ny, d->pitch, d->plane,
                                              scratch, d->stream);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(body, scratch, 4 * (size_t)n, cudaMemcpyDeviceToHost, d->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(d->stream);
    if (e != cudaSuccess || check_pairs(d) != LE2D_OK) {
      if (e != cudaSuccess) record(d, LE2D_ECUDA, "le_save_task", e);
      free(body);
      return 1;
    }
  } else {
    if (d && ensure_host_current(d, t)) {
      free(body);
      return 1;
    }
    for (long long q = 0; q < n; q++) {
      const real vx = t->stype == ST_AOS ? t->grid[q * 5 + 0] : t->grid[q];
      const real vy = t->stype == ST_AOS ? t->grid[q * 5 + 1] : t->grid[n + q];
      const float v = sqrt(vx * vx + vy * vy);
      unsigned char b[4];
      memcpy(b, &v, 4);
      body[4 * q + 0] = b[3];
      body[4 * q + 1] = b[2];
      body[4 * q + 2] = b[1];
      body[4 * q + 3] = b[0];
    }
  }
  FILE* fp = fopen(file, "w");
  if (!fp) {
    perror("Failed to open file");
    free(body);
    return 1;
  }
  fprintf(fp, "# vtk DataFile Version 3.0\n");
  fprintf(fp, "Created by le_save_task\n");
  fprintf(fp, "BINARY\n");
  fprintf(fp, "DATASET STRUCTURED_POINTS\n");
  fprintf(fp, "DIMENSIONS %d %d 1\n", t->n.x, t->n.y);
  fprintf(fp, "SPACING %f %f 0.0\n", t->h.x, t->h.y);
  fprintf(fp, "ORIGIN 0.0 0.0 0.0\n");
  fprintf(fp, "POINT_DATA %d\n", t->n.x * t->n.y);
  fprintf(fp, "SCALARS v float 1\n");
  fprintf(fp, "LOOKUP_TABLE v_table\n");
  fwrite(body, 1, 4 * (size_t)n, fp);
  free(body);
  fclose(fp);
  return 0;
}

void le_step(le_task* task) { run_steps(task, 1, false, nullptr); }

void le_step_soa(le_task* task) { run_steps(task, 1, true, nullptr); }

int le2d_step_n(le_task* task, int nsteps) {
  return run_steps(task, nsteps, task && task->stype == ST_SOA, nullptr);
}

int le2d_step_n_timed(le_task* task, int nsteps, float* ms) {
  if (!ms) return LE2D_EINVAL;
  return run_steps(task, nsteps, task && task->stype == ST_SOA, ms);
}

int le2d_last_error(const le_task* task) {
  DevTask* d = lookup(task);
  return d ? d->err : LE2D_ENOTASK;
}

int le2d_clear_error(le_task* task) {
  DevTask* d = lookup(task);
  if (!d) return LE2D_ENOTASK;
  d->err = LE2D_OK;
  return LE2D_OK;
}

int le2d_sync_host(le_task* task) {
  DevTask* d = lookup_sync(task);
  if (!d) return LE2D_ENOTASK;
  return ensure_host_current(d, task);
}

int le2d_sync_device(le_task* task) {
  DevTask* d = lookup_sync(task);
  if (!d) return LE2D_ENOTASK;
  d->host_newer = true;
  d->dev_newer = false;
  return ensure_device_current(d, task);
}

int le2d_upload(le_task* task, const real* src) {
  DevTask* d = lookup_sync(task);
  if (!d) return LE2D_ENOTASK;
  if (!src) return record(d, LE2D_EINVAL, "le2d_upload: NULL source");
  if (!d->has_device) return record(d, LE2D_ENODEV, "le2d_upload");
  const int rc = upload_raw(d, src, task->stype == ST_AOS);
  if (rc) return rc;
  d->host_newer = false;
  d->dev_newer = true;
  return LE2D_OK;
}

int le2d_download(le_task* task, real* dst) {
  DevTask* d = lookup_sync(task);
  if (!d) return LE2D_ENOTASK;
  if (!dst) return record(d, LE2D_EINVAL, "le2d_download: NULL destination");
  if (d->host_newer) {
    memcpy(dst, task->grid, sizeof(le_node) * (size_t)d->nx * d->ny);
    return LE2D_OK;
  }
  if (!d->has_device) return record(d, LE2D_ENODEV, "le2d_download");
  return download_raw(d, dst, task->stype == ST_AOS);
}

void* le2d_host_alloc(size_t bytes) {
  void* p = nullptr;
  if (device_count() == 0 || cudaHostAlloc(&p, bytes, cudaHostAllocDefault) != cudaSuccess) {
    cudaGetLastError();
    return nullptr;
  }
  return p;
}

void le2d_host_free(void* p) {
  if (p) cudaFreeHost(p);
}

int le2d_wait(le_task* task) {
  DevTask* d = lookup_sync(task);
  if (!d) return LE2D_ENOTASK;
  if (!d->has_device) return LE2D_OK;
  cudaError_t e = cudaStreamSynchronize(d->stream);
  return e == cudaSuccess ? check_pairs(d) : record(d, LE2D_ECUDA, "wait", e);
}

int le2d_set_method(le_task* task, int method) {
  DevTask* d = lookup_sync(task);
  if (!d) return LE2D_ENOTASK;
  if (method != LE2D_METHOD_FUSED && method != LE2D_METHOD_SPLIT) return LE2D_EINVAL;
  d->method = method;
  return LE2D_OK;
}

int le2d_set_variant(le_task* task, int variant, int seg_len) {
  DevTask* d = lookup_sync(task);
  if (!d) return LE2D_ENOTASK;
  if (variant < -1 || variant >= le2d::fused_variant_count<T>() || seg_len < 0) return LE2D_EINVAL;
  if (!d->has_device) return LE2D_ENODEV;
  replan(d, variant < 0 ? default_variant() : variant, seg_len);
  return LE2D_OK;
}

int le2d_autotune(int nx, int ny, int* out_plan, double* nu_per_s) {
  if (nx < 3 || ny < 3) return LE2D_EINVAL;
  if (device_count() == 0) return LE2D_ENODEV;
  Tuned t;
  const int rc = tune_size(nx, ny, &t);
  if (rc) return rc;
  {
    std::lock_guard<std::mutex> lk(g_tune_mu);
    g_tuned[size_class(nx, ny)] = t;
  }
  if (nu_per_s) *nu_per_s = t.nu_s;
  if (out_plan) {
    int dev = 0;
    cudaGetDevice(&dev);
    le2d::FusedPlan p = le2d::plan_fused<T>(nx, ny, t.variant,
                                            le2d::fused_resident_warps<T>(dev, t.variant), kMinSeg);
    out_plan[0] = t.variant;
    out_plan[1] = p.lanes;
    out_plan[2] = t.seg_len > 0 ? (t.seg_len < ny ? t.seg_len : ny) : p.seg_len;
    out_plan[3] = p.nstrips;
    out_plan[4] = p.nstrips * ((ny + out_plan[2] - 1) / out_plan[2]);
    const int tpb = p.threads / 32 / p.warps_per_task;  // tiles per block
    out_plan[5] = (out_plan[4] + tpb - 1) / tpb;
    out_plan[6] = p.depth;
    out_plan[7] = p.warps_per_task;
  }
  return LE2D_OK;
}

int le2d_autotune_reset(void) {
  std::lock_guard<std::mutex> lk(g_tune_mu);
  g_tuned.clear();
  return LE2D_OK;
}

int le2d_get_plan(const le_task* task, int* out) {
  DevTask* d = lookup(task);
  if (!d) return LE2D_ENOTASK;
  if (!out) return LE2D_EINVAL;
  out[0] = d->plan.variant;
  out[1] = d->plan.lanes;
  out[2] = d->plan.seg_len;
  out[3] = d->plan.nstrips;
  out[4] = d->plan.ntasks;
  out[5] = d->plan.blocks;
  out[6] = d->plan.depth;
  out[7] = d->plan.warps_per_task;
  return LE2D_OK;
}

int le2d_launch_parts(const le_task* task, int* parts) {
  DevTask* d = lookup(task);
  if (!d) return LE2D_ENOTASK;
  if (!parts) return LE2D_EINVAL;
  *parts = d->halves ? 3 : 1;
  return LE2D_OK;
}

int le2d_sim_time(const le_task* task, double* t, long long* steps) {
  DevTask* d = lookup(task);
  if (!d) return LE2D_ENOTASK;
  if (t) *t = d->sim_time;
  if (steps) *steps = d->steps;
  return LE2D_OK;
}

int le2d_diagnostics(le_task* task, le2d_diag_t* out) {
  DevTask* d = lookup_sync(task);
  if (!d) return LE2D_ENOTASK;
  if (!out) return LE2D_EINVAL;
  int rc = ensure_device_current(d, task);
  if (rc) return rc;
  const double rho = task->mat.rho, c1 = task->mat.c1, c2 = task->mat.c2;
  const double mu = rho * c2 * c2, la = rho * c1 * c1 - 2.0 * mu;
  const double a_nn = (la + 2.0 * mu) / (8.0 * mu * (la + mu));
  const double a_xy = -2.0 * la / (8.0 * mu * (la + mu));
  const double a_s = 1.0 / (2.0 * mu);
  double h[11];
  cudaError_t e = cudaMemsetAsync(d->d_diag, 0, 11 * sizeof(double), d->stream);
  if (e == cudaSuccess)
    e = le2d::launch_diag<T>(d->buf[d->cur], d->nx, d->ny, d->pitch, d->plane, rho, a_nn, a_xy, a_s,
                             d->d_diag, d->stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(h, d->d_diag, sizeof(h), cudaMemcpyDeviceToHost, d->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(d->stream);
  if (e != cudaSuccess) return record(d, LE2D_ECUDA, "diagnostics", e);
  out->energy = h[0] * (double)task->h.x * (double)task->h.y;
  for (int k = 0; k < 5; ++k) {
    out->sumsq[k] = h[1 + k];
    out->maxabs[k] = h[6 + k];
  }
  return LE2D_OK;
}

}  // extern "C"

namespace {

// Rows [row0, row0 + nrows) of the task's state <-> a caller's device buffer laid out
// [field][row][nx], on the caller's stream `stream`, ordered with the task's stream both ways
// (events), so a caller can hand the rows to a collective on its own stream.
int copy_rows(le_task* task, int row0, int nrows, T* dev_buf, void* stream, bool out) {
  DevTask* d = lookup_sync(task);
  if (!d) return LE2D_ENOTASK;
  const char* what = out ? "le2d_rows_out" : "le2d_rows_in";
  if (!dev_buf || nrows < 0 || row0 < 0 || row0 + nrows > d->ny) return record(d, LE2D_EINVAL, what);
  int rc = ensure_device_current(d, task);
  if (rc) return rc;
  if (nrows == 0) return LE2D_OK;
  const cudaStream_t s = (cudaStream_t)stream;
  cudaError_t e = cudaEventRecord(d->ev[0], d->stream);
  if (e == cudaSuccess) e = cudaStreamWaitEvent(s, d->ev[0], 0);
  for (int k = 0; k < 5 && e == cudaSuccess; ++k) {
    T* state = d->buf[d->cur] + k * d->plane + (long long)row0 * d->pitch;
    T* flat = dev_buf + (size_t)k * nrows * d->nx;
    if (out)
      e = cudaMemcpy2DAsync(flat, sizeof(T) * d->nx, state, sizeof(T) * d->pitch, sizeof(T) * d->nx, nrows,
                            cudaMemcpyDeviceToDevice, s);
    else
      e = cudaMemcpy2DAsync(state, sizeof(T) * d->pitch, flat, sizeof(T) * d->nx, sizeof(T) * d->nx, nrows,
                            cudaMemcpyDeviceToDevice, s);
  }
  if (e == cudaSuccess) e = cudaEventRecord(d->ev[1], s);
  if (e == cudaSuccess) e = cudaStreamWaitEvent(d->stream, d->ev[1], 0);
  if (e != cudaSuccess) return record(d, LE2D_ECUDA, what, e);
  if (!out) d->dev_newer = true;
  return LE2D_OK;
}

}  // namespace

extern "C" {

int le2d_check_violations(unsigned long long* count) {
#ifdef LE2D_CHECK
  const unsigned long long a = le2d::check_violations_fused(), b = le2d::check_violations_batch();
  if (count) *count = a == ~0ULL || b == ~0ULL ? ~0ULL : a + b;
  return 1;
#else
  if (count) *count = 0;
  return 0;
#endif
}

int le2d_rows_out(le_task* task, int row0, int nrows, real* dev_buf, void* stream) {
  return copy_rows(task, row0, nrows, dev_buf, stream, true);
}

int le2d_rows_in(le_task* task, int row0, int nrows, const real* dev_buf, void* stream) {
  return copy_rows(task, row0, nrows, const_cast<real*>(dev_buf), stream, false);
}

int le2d_device_layout(const le_task* task, long long* pitch_elems, long long* plane_elems) {
  DevTask* d = lookup(task);
  if (!d) return LE2D_ENOTASK;
  if (pitch_elems) *pitch_elems = d->pitch;
  if (plane_elems) *plane_elems = d->plane;
  return LE2D_OK;
}

}  // extern "C"
