// Batched solves: instance states in a device arena, per-window work lists for the
// persistent kernel (batch.cu), CUDA-graph capture of the window loop, read-back.
#include <algorithm>
#include <type_traits>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <iterator>
#include <mutex>

#include "consts.h"
#include "engine.h"

namespace le2d {

// ---------------------------------------------------------------- Arena

Arena::Arena(size_t capacity) {
  capacity = capacity / 256 * 256;
  if (capacity == 0 || cudaMalloc(&base_, capacity) != cudaSuccess) {
    cudaGetLastError();
    base_ = nullptr;
    return;
  }
  cap_ = capacity;
  free_[0] = capacity;
}

Arena::~Arena() {
  if (base_) cudaFree(base_);
}

size_t Arena::alloc(size_t bytes) {
  bytes = (bytes + 255) / 256 * 256;
  if (bytes == 0) bytes = 256;
  for (auto it = free_.begin(); it != free_.end(); ++it) {
    if (it->second < bytes) continue;
    const size_t off = it->first, sz = it->second;
    free_.erase(it);
    if (sz > bytes) free_[off + bytes] = sz - bytes;
    live_[off] = bytes;
    used_ += bytes;
    return off;
  }
  return SIZE_MAX;
}

void Arena::free(size_t off) {
  auto it = live_.find(off);
  if (it == live_.end()) return;
  size_t sz = it->second;
  live_.erase(it);
  used_ -= sz;
  auto next = free_.lower_bound(off);
  if (next != free_.end() && off + sz == next->first) {
    sz += next->second;
    next = free_.erase(next);
  }
  if (next != free_.begin()) {
    auto prev = std::prev(next);
    if (prev->first + prev->second == off) {
      prev->second += sz;
      return;
    }
  }
  free_[off] = sz;
}

// ---------------------------------------------------------------- Engine

template <typename T>
StepConsts<T> problem_consts(const le2d_problem& p) {
  le_material m;
  le_init_material(p.c1, p.c2, p.rho, &m);
  le_vec2 h;
  h.x = p.hx;
  h.y = p.hy;
  return make_consts(p.dt, h, m);
}

template <typename T>
Engine<T>::Engine(size_t budget) {
  size_t freeb = 0, total = 0;
  if (cudaMemGetInfo(&freeb, &total) != cudaSuccess) {
    cudaGetLastError();
    return;
  }
  const size_t reserve = (size_t)512 << 20;  // scratch and other users of the device
  const size_t avail = freeb > reserve ? freeb - reserve : 0;
  if (budget == 0 || budget > avail) budget = (size_t)(0.9 * (double)avail);
  arena_ = new Arena(budget);
  if (cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking) != cudaSuccess) stream_ = nullptr;
  if (cudaStreamCreateWithFlags(&copy_, cudaStreamNonBlocking) != cudaSuccess) {
    if (stream_) cudaStreamDestroy(stream_);
    stream_ = copy_ = nullptr;
  }
  cudaEventCreate(&ev_[0]);
  cudaEventCreate(&ev_[1]);
  if (cudaMalloc(&d_diag_, 16 * sizeof(double)) != cudaSuccess) d_diag_ = nullptr;
  int dev = 0;
  cudaGetDevice(&dev);
  resident_blocks_ = batch_resident_blocks<T>(dev);
  // Test hook for the bounded-wait path: in the engine's first window, tile k of the work
  // list never publishes its first step, so its instance fails (LE2D_ETIMEOUT) while the
  // other instances finish.
  if (const char* s = getenv("LE2D_TEST_STALL_TILE")) stall_tile_ = atoi(s);
}

template <typename T>
Engine<T>::~Engine() {
  if (stream_) cudaStreamSynchronize(stream_);
  if (copy_) cudaStreamSynchronize(copy_);
  delete arena_;
  cudaFree(d_insts_);
  cudaFree(d_tiles_);
  cudaFree(d_items_);
  cudaFree(d_done_);
  cudaFree(d_ctl_);
  cudaFree(d_diag_);
  if (ev_[0]) cudaEventDestroy(ev_[0]);
  if (ev_[1]) cudaEventDestroy(ev_[1]);
  if (stream_) cudaStreamDestroy(stream_);
  if (copy_) cudaStreamDestroy(copy_);
}

template <typename T>
size_t Engine<T>::footprint(const le2d_problem& p) {
  if (p.nx < 1 || p.ny < 1) return 0;
  const long long pitch = row_pitch_elems(p.nx);
  size_t b = (sizeof(T) * 2 * 5 * (size_t)pitch * (size_t)p.ny + 255) / 256 * 256 + 256;  // + failure word
  if (p.receiver_row >= 0 && p.receiver_every > 0)
    b += (sizeof(T) * 2 * (size_t)pitch * (size_t)(p.steps / p.receiver_every) + 255) / 256 * 256;
  return b;
}

template <typename T>
int Engine<T>::set_seg_len(int rows) {
  if (rows < 1) return LE2D_EINVAL;
  seg_len_ = rows;
  seg_set_ = true;
  return LE2D_OK;
}

template <typename T>
int Engine<T>::set_depth(int depth) {
  if (depth < 1 || depth > 2) return LE2D_EINVAL;
  depth_set_ = depth;
  return LE2D_OK;
}

// ---------------------------------------------------------------- batched autotuner

namespace {
std::mutex g_bt_mu;
std::map<std::pair<int, int>, BatchTuned> g_bt;

int ceil_log2(int n) {
  int k = 0;
  while ((1 << k) < n) ++k;
  return k;
}
}  // namespace

bool batch_tuned(int nx, int ny, BatchTuned* out) {
  std::lock_guard<std::mutex> lk(g_bt_mu);
  auto it = g_bt.find({ceil_log2(nx), ceil_log2(ny)});
  if (it == g_bt.end()) return false;
  *out = it->second;
  return true;
}

void batch_tune_reset() {
  std::lock_guard<std::mutex> lk(g_bt_mu);
  g_bt.clear();
}

// Times the batched kernel on copies of a scratch nx x ny problem (a disk of radius
// min(nx,ny)/4 on a zero field, c1 = 2, c2 = 1, rho = 1, Courant number 0.5; enough copies
// for ~24 M nodes, at most 256) for every tile height and steps per work item, and keeps
// the fastest for the size class.
template <typename T>
int batch_autotune(int nx, int ny, BatchTuned* best) {
  le2d_problem p;
  std::memset(&p, 0, sizeof(p));
  p.nx = nx;
  p.ny = ny;
  p.hx = p.hy = 1;
  p.dt = (real)0.25;
  p.c1 = 2;
  p.c2 = 1;
  p.rho = 1;
  p.stype = ST_AOS;
  p.receiver_row = -1;
  p.receiver_every = 1;
  const double nodes = (double)nx * ny;
  const int copies = (int)std::max(1.0, std::min(256.0, std::ceil(24e6 / nodes)));
  int steps = (int)std::min(512.0, std::max(8.0, 4e9 / (copies * nodes)));
  steps += steps & 1;
  p.steps = steps;
  const T disk[4] = {(T)(nx / 2), (T)(ny / 2), (T)(std::min(nx, ny) / 4), (T)1};
  const size_t budget = Engine<T>::footprint(p) * copies + ((size_t)64 << 20);
  const int segs[] = {16, 32, 64, 128, 256};
  best->nu_s = -1.0;
  bool warm = false;
  for (int d = 1; d <= batch_depth<T>(); ++d) {
    for (int seg : segs) {
      if (seg > ny && seg != segs[0]) continue;
      for (int rep = 0; rep < (warm ? 1 : 2); ++rep) {  // the first trial runs twice (warm-up)
        Engine<T> e(budget);
        if (!e.ok()) return LE2D_ENOMEM;
        e.set_seg_len(seg);
        e.set_depth(d);
        for (int k = 0; k < copies; ++k) {
          const int id = e.add(p, nullptr, 1, disk);
          if (id < 0) return -id;
        }
        float ms = 0.0f;
        const int rc = e.run_all(steps, &ms);
        if (rc) return rc;
        const double nus = copies * nodes * steps / (ms * 1e-3);
        if (rep == (warm ? 0 : 1) && nus > best->nu_s) {
          best->nu_s = nus;
          best->seg_len = seg;
          best->depth = d;
        }
      }
      warm = true;
    }
  }
  std::lock_guard<std::mutex> lk(g_bt_mu);
  g_bt[{ceil_log2(nx), ceil_log2(ny)}] = *best;
  return LE2D_OK;
}

// Validation, arena blocks (both state buffers and the failure word; receiver samples),
// constants and tiles of a new instance.  Returns LE2D_OK or -LE2D_E*.
template <typename T>
int Engine<T>::alloc_instance(const le2d_problem& p, Inst& in) {
  if (!ok()) return -LE2D_ENODEV;
  if (p.nx < 3 || p.ny < 3 || p.steps < 0 || !(p.hx > 0) || !(p.hy > 0) || !(p.dt > 0) ||
      !(p.c1 > 0) || !(p.c2 > 0) || !(p.rho > 0) || (p.stype != ST_AOS && p.stype != ST_SOA) ||
      p.receiver_row >= p.ny || (p.receiver_row >= 0 && p.receiver_every < 1))
    return -LE2D_EINVAL;
  // CFL: the Courant numbers must not exceed 1 (the scheme is stable for k <= 1).
  if ((double)p.dt * p.c1 > (double)std::min(p.hx, p.hy)) return -LE2D_EINVAL;
  in.p = p;
  in.pitch = row_pitch_elems(p.nx);
  in.plane = in.pitch * p.ny;
  const size_t sbytes = sizeof(T) * 2 * 5 * (size_t)in.plane;
  in.state_off = arena_->alloc(sbytes + 256);
  if (in.state_off == SIZE_MAX) return -LE2D_EBUDGET;
  if (p.receiver_row >= 0) {
    in.nsamples = p.steps / p.receiver_every;
    if (in.nsamples > 0) {
      in.trace_off = arena_->alloc(sizeof(T) * 2 * (size_t)in.pitch * in.nsamples);
      if (in.trace_off == SIZE_MAX) {
        arena_->free(in.state_off);
        return -LE2D_EBUDGET;
      }
      in.trace = reinterpret_cast<T*>(arena_->base() + in.trace_off);
    }
  }
  in.buf[0] = reinterpret_cast<T*>(arena_->base() + in.state_off);
  in.buf[1] = in.buf[0] + 5 * in.plane;
  in.fail = reinterpret_cast<int*>(arena_->base() + in.state_off + sbytes);
  in.c = problem_consts<T>(p);
  // Tile height and steps per work item: explicit (autotuner trials), else the autotuner's
  // table for the size class (LE2D_AUTOTUNE=1 tunes a class on first use), else defaults.
  int seg = seg_len_, depth = batch_depth<T>();
  if (!seg_set_ && !depth_set_ && use_tuned_) {
    BatchTuned bt;
    bool have = batch_tuned(p.nx, p.ny, &bt);
    const char* a = getenv("LE2D_AUTOTUNE");
    if (!have && a && atoi(a) != 0) have = batch_autotune<T>(p.nx, p.ny, &bt) == LE2D_OK;
    if (have) {
      seg = bt.seg_len;
      depth = bt.depth;
    }
  }
  if (depth_set_) depth = std::min(depth_set_, batch_depth<T>());
  // le_step_soa's far end is not a clamp: its instances advance one step per work item
  in.depth = p.stype == ST_AOS ? depth : 1;
  // one- and two-step tiles have the same strips at the two-step kernel's 4 columns per
  // lane (one halo lane per side for either)
  static_assert(strip_cols(4) == strip_cols2(4), "strip widths of one and two steps");
  const int out = strip_cols(batch_lanes<T>());
  in.nstrips = (p.nx + out - 1) / out;
  in.seg_len = std::min(seg, p.ny);
  in.nsegs = (p.ny + in.seg_len - 1) / in.seg_len;
  in.live = true;
  return LE2D_OK;
}

template <typename T>
int Engine<T>::add(const le2d_problem& p, const T* init, int ndisks, const T* disks) {
  if (ndisks < 0 || (ndisks > 0 && !disks)) return -LE2D_EINVAL;
  Inst in;
  int rc = alloc_instance(p, in);
  if (rc) return rc;
  const size_t sbytes = sizeof(T) * 2 * 5 * (size_t)in.plane;
  cudaError_t e = cudaMemsetAsync(in.buf[0], 0, sbytes + 256, stream_);  // states, failure word
  if (e == cudaSuccess && in.trace)
    e = cudaMemsetAsync(in.trace, 0, sizeof(T) * 2 * (size_t)in.pitch * in.nsamples, stream_);
  if (e == cudaSuccess && init) {
    const size_t bytes = sizeof(T) * 5 * (size_t)p.nx * p.ny;
    e = cudaMemcpyAsync(in.buf[1], init, bytes, cudaMemcpyHostToDevice, stream_);
    if (e == cudaSuccess)
      e = launch_pack<T>(in.buf[1], in.buf[0], p.nx, p.ny, in.pitch, in.plane, p.stype == ST_AOS,
                         stream_);
    if (e == cudaSuccess) e = cudaStreamSynchronize(stream_);  // `init` may be freed on return
  }
  for (int k = 0; k < ndisks && e == cudaSuccess && !init; ++k)
    e = launch_set_ball<T>(in.buf[0], p.nx, p.ny, in.pitch, in.plane, p.hx, p.hy, disks[4 * k],
                           disks[4 * k + 1], disks[4 * k + 2], disks[4 * k + 3], stream_);
  if (e != cudaSuccess) {
    fprintf(stderr, "le2d: batch add: %s\n", cudaGetErrorString(e));
    arena_->free(in.state_off);
    if (in.trace) arena_->free(in.trace_off);
    return -LE2D_ECUDA;
  }
  insts_.push_back(in);
  return (int)insts_.size() - 1;
}

template <typename T>
int Engine<T>::add_async(const le2d_problem& p, const T* init, int ndisks, const T* disks) {
  if (ndisks < 0 || (ndisks > 0 && !disks)) return -LE2D_EINVAL;
  Inst in;
  int rc = alloc_instance(p, in);
  if (rc) return rc;
  cudaError_t e = cudaSuccess;
  if (init) {  // the host state into the second buffer, beside the window in flight
    e = cudaMemcpyAsync(in.buf[1], init, sizeof(T) * 5 * (size_t)p.nx * p.ny, cudaMemcpyHostToDevice,
                        copy_);
    if (e == cudaSuccess) e = cudaStreamSynchronize(copy_);  // `init` may be freed on return
    in.has_init = true;
  } else {
    in.disks.assign(disks, disks + 4 * (size_t)ndisks);
  }
  if (e != cudaSuccess) {
    fprintf(stderr, "le2d: batch add: %s\n", cudaGetErrorString(e));
    arena_->free(in.state_off);
    if (in.trace) arena_->free(in.trace_off);
    return -LE2D_ECUDA;
  }
  in.prologue = true;
  insts_.push_back(in);
  return (int)insts_.size() - 1;
}

// Initial conditions of instances added by add_async: state and failure word cleared, the
// uploaded host state packed (or the disks set) -- small kernels queued just before a window.
template <typename T>
int Engine<T>::apply_prologues() {
  cudaError_t e = cudaSuccess;
  for (Inst& in : insts_) {
    if (!in.live || !in.prologue) continue;
    const size_t bytes = sizeof(T) * 5 * (size_t)in.plane;
    e = cudaMemsetAsync(in.buf[0], 0, bytes, stream_);
    if (e == cudaSuccess) e = cudaMemsetAsync(in.fail, 0, 256, stream_);
    if (e == cudaSuccess && in.trace)
      e = cudaMemsetAsync(in.trace, 0, sizeof(T) * 2 * (size_t)in.pitch * in.nsamples, stream_);
    if (e == cudaSuccess && in.has_init)
      e = launch_pack<T>(in.buf[1], in.buf[0], in.p.nx, in.p.ny, in.pitch, in.plane,
                         in.p.stype == ST_AOS, stream_);
    for (size_t k = 0; e == cudaSuccess && 4 * k < in.disks.size(); ++k)
      e = launch_set_ball<T>(in.buf[0], in.p.nx, in.p.ny, in.pitch, in.plane, in.p.hx, in.p.hy,
                             in.disks[4 * k], in.disks[4 * k + 1], in.disks[4 * k + 2],
                             in.disks[4 * k + 3], stream_);
    if (e != cudaSuccess) break;
    in.prologue = false;
    in.disks.clear();
    in.disks.shrink_to_fit();
  }
  if (e != cudaSuccess) fprintf(stderr, "le2d: initial condition: %s\n", cudaGetErrorString(e));
  return e == cudaSuccess ? LE2D_OK : LE2D_ECUDA;
}

// Reads the failure words of these instances (after a launch that reported failures).
template <typename T>
int Engine<T>::read_failures(const std::vector<int>& ids) {
  for (int id : ids) {
    Inst& in = insts_[id];
    int f = 0;
    if (cudaMemcpy(&f, in.fail, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess) return LE2D_ECUDA;
    if (f != 0) in.failed = true;
  }
  return LE2D_OK;
}

template <typename T>
typename Engine<T>::Window Engine<T>::plan_window(int window, const std::vector<long long>& done,
                                                  const std::vector<int>& cur) const {
  Window w;
  std::vector<std::pair<int, int>> order;  // (work-item steps in window, id)
  std::vector<int> steps_of(insts_.size(), 0);
  for (int id = 0; id < (int)insts_.size(); ++id) {
    const Inst& in = insts_[id];
    if (!in.live || in.failed) continue;
    const long long left = in.p.steps - done[id];
    if (left <= 0) continue;
    steps_of[id] = (int)std::min<long long>(left, window);
    order.push_back({(steps_of[id] + in.depth - 1) / in.depth, id});
  }
  std::stable_sort(order.begin(), order.end(),
                   [](const std::pair<int, int>& a, const std::pair<int, int>& b) {
                     return a.first > b.first;
                   });
  int tile_base = 0;
  for (size_t k = 0; k < order.size(); ++k) {
    const Inst& in = insts_[order[k].second];
    BatchInst<T> b;
    b.buf[0] = in.buf[0];
    b.buf[1] = in.buf[1];
    b.nx = in.p.nx;
    b.ny = in.p.ny;
    b.pitch = in.pitch;
    b.plane = in.plane;
    b.c = in.c;
    b.yq = YPairs{};
    if constexpr (std::is_same<T, float>::value) b.yq = make_ypairs(in.c.y);
    b.far_rot = in.p.stype == ST_SOA;
    b.nstrips = in.nstrips;
    b.nsegs = in.nsegs;
    b.seg_len = in.seg_len;
    b.tile_base = tile_base;
    b.parity = cur[order[k].second];
    b.steps = steps_of[order[k].second];
    b.depth = in.depth;
    b.abs_step0 = done[order[k].second];
    b.trace = in.trace;
    b.trace_row = in.trace ? in.p.receiver_row : -1;
    b.trace_every = in.trace ? in.p.receiver_every : 1;
    b.fail = in.fail;
    w.insts.push_back(b);
    w.inst_ids.push_back(order[k].second);
    w.inst_steps.push_back(steps_of[order[k].second]);
    w.inst_items.push_back(order[k].first);
    for (int s = 0; s < in.nsegs; ++s)
      for (int st = 0; st < in.nstrips; ++st) w.tiles.push_back(BatchTile{(int)k, st, s, 0});
    tile_base += in.nstrips * in.nsegs;
  }
  w.steps = order.empty() ? 0 : order.front().first;
  w.step_items.assign(w.steps + 1, 0);
  size_t active = order.size();  // instances with steps in window > r form a prefix
  for (int r = 0; r < w.steps; ++r) {
    while (active > 0 && order[active - 1].first <= r) --active;
    const long long tiles = active == 0 ? 0 : w.insts[active - 1].tile_base +
                                                  (long long)w.insts[active - 1].nstrips *
                                                      w.insts[active - 1].nsegs;
    w.step_items[r + 1] = w.step_items[r] + tiles;
  }
  return w;
}

template <typename T>
int Engine<T>::ensure_scratch(size_t ni, size_t nt, size_t nitems, size_t ndone, size_t nctl) {
  auto grow = [](auto*& p, size_t& cap, size_t need, size_t elem) -> bool {
    if (need <= cap) return true;
    cudaFree(p);
    p = nullptr;
    size_t n = std::max(need, cap * 2);
    if (cudaMalloc((void**)&p, n * elem) != cudaSuccess) {
      cudaGetLastError();
      cap = 0;
      return false;
    }
    cap = n;
    return true;
  };
  bool ok = grow(d_insts_, cap_insts_, ni, sizeof(BatchInst<T>)) &&
            grow(d_tiles_, cap_tiles_, nt, sizeof(BatchTile)) &&
            grow(d_items_, cap_items_, nitems, sizeof(long long)) &&
            grow(d_done_, cap_done_, ndone, sizeof(int)) && grow(d_ctl_, cap_ctl_, nctl, sizeof(BatchCtl));
  return ok ? LE2D_OK : LE2D_ENOMEM;
}

template <typename T>
int Engine<T>::launch_window(const Window& w, size_t io, size_t to, size_t so, size_t doff,
                             size_t co) {
  cudaError_t e = cudaMemsetAsync(d_done_ + doff, 0, sizeof(int) * std::max<size_t>(w.tiles.size(), 1), stream_);
  if (e == cudaSuccess) e = cudaMemsetAsync(d_ctl_ + co, 0, sizeof(BatchCtl), stream_);
  if (e == cudaSuccess)
    e = launch_batch<T>(d_insts_ + io, d_tiles_ + to, d_items_ + so, w.steps, w.step_items.back(),
                        d_done_ + doff, d_ctl_ + co, wait_ns_, stall_tile_ + 1, resident_blocks_,
                        stream_);
  stall_tile_ = -1;  // the hook stalls one window
  return e == cudaSuccess ? LE2D_OK : LE2D_ECUDA;
}

template <typename T>
int Engine<T>::begin_window(int window) {
  if (!ok()) return LE2D_ENODEV;
  if (window < 1) return LE2D_EINVAL;
  if (in_flight_) return LE2D_ESTATE;
  int rc = apply_prologues();
  if (rc) return rc;
  std::vector<long long> done(insts_.size());
  std::vector<int> cur(insts_.size());
  for (size_t i = 0; i < insts_.size(); ++i) {
    done[i] = insts_[i].done_steps;
    cur[i] = insts_[i].cur;
  }
  win_ = plan_window(window, done, cur);
  if (win_.steps == 0) return LE2D_OK;
  const Window& w = win_;
  rc = ensure_scratch(w.insts.size(), w.tiles.size(), w.step_items.size(), w.tiles.size(), 1);
  if (rc) return rc;
  cudaError_t e = cudaMemcpyAsync(d_insts_, w.insts.data(), sizeof(BatchInst<T>) * w.insts.size(),
                                  cudaMemcpyHostToDevice, stream_);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(d_tiles_, w.tiles.data(), sizeof(BatchTile) * w.tiles.size(),
                        cudaMemcpyHostToDevice, stream_);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(d_items_, w.step_items.data(), sizeof(long long) * w.step_items.size(),
                        cudaMemcpyHostToDevice, stream_);
  if (e != cudaSuccess) return LE2D_ECUDA;
  rc = launch_window(w, 0, 0, 0, 0, 0);
  if (rc) return rc;
  // final fields of the instances this window finishes, unpacked into their idle buffer
  // right after it, so that reading them back needs no kernel beside the next window
  for (size_t k = 0; k < w.inst_ids.size() && e == cudaSuccess; ++k) {
    Inst& in = insts_[w.inst_ids[k]];
    if (in.done_steps + w.inst_steps[k] < in.p.steps) continue;
    const int c = in.cur ^ (w.inst_items[k] & 1);
    e = launch_unpack<T>(in.buf[c], in.buf[c ^ 1], in.p.nx, in.p.ny, in.pitch, in.plane,
                         in.p.stype == ST_AOS, stream_);
    in.unpacked = true;
  }
  if (e != cudaSuccess) return LE2D_ECUDA;
  in_flight_ = true;
  return LE2D_OK;
}

template <typename T>
int Engine<T>::end_window() {
  if (!in_flight_) return LE2D_OK;
  in_flight_ = false;
  const Window& w = win_;
  BatchCtl ctl;
  cudaError_t e = cudaMemcpyAsync(&ctl, d_ctl_, sizeof(ctl), cudaMemcpyDeviceToHost, stream_);
  if (e == cudaSuccess) e = cudaStreamSynchronize(stream_);
  if (e != cudaSuccess) return LE2D_ECUDA;
  if (ctl.status != 0) {  // a wait inside a warp pair gave up: the launch ended early
    for (int id : w.inst_ids) insts_[id].failed = true;
    return LE2D_ETIMEOUT;
  }
  if (ctl.failed != 0 && read_failures(w.inst_ids) != LE2D_OK) return LE2D_ECUDA;
  for (size_t k = 0; k < w.inst_ids.size(); ++k) {
    Inst& in = insts_[w.inst_ids[k]];
    if (in.failed) continue;
    in.done_steps += w.inst_steps[k];
    in.cur ^= w.inst_items[k] & 1;  // each work-item step writes the other buffer
    node_updates_ += (long long)in.p.nx * in.p.ny * w.inst_steps[k];
  }
  return LE2D_OK;
}

template <typename T>
int Engine<T>::run_window(int window) {
  const int rc = begin_window(window);
  return rc ? rc : end_window();
}

template <typename T>
int Engine<T>::run_all(int window, float* ms) {
  if (!ok()) return LE2D_ENODEV;
  if (window < 1) return LE2D_EINVAL;
  if (in_flight_) return LE2D_ESTATE;
  if (apply_prologues() != LE2D_OK) return LE2D_ECUDA;
  std::vector<long long> done(insts_.size());
  std::vector<int> cur(insts_.size());
  for (size_t i = 0; i < insts_.size(); ++i) {
    done[i] = insts_[i].done_steps;
    cur[i] = insts_[i].cur;
  }
  std::vector<Window> ws;
  size_t ni = 0, nt = 0, nitems = 0;
  while (true) {
    Window w = plan_window(window, done, cur);
    if (w.steps == 0) break;
    for (size_t k = 0; k < w.inst_ids.size(); ++k) {
      done[w.inst_ids[k]] += w.inst_steps[k];
      cur[w.inst_ids[k]] ^= w.inst_items[k] & 1;
    }
    ni += w.insts.size();
    nt += w.tiles.size();
    nitems += w.step_items.size();
    ws.push_back(std::move(w));
  }
  if (ws.empty()) {
    if (ms) *ms = 0.0f;
    return LE2D_OK;
  }
  int rc = ensure_scratch(ni, nt, nitems, nt, ws.size());
  if (rc) return rc;
  // upload every window's lists, then capture the window loop in one graph
  std::vector<size_t> io(ws.size()), to(ws.size()), so(ws.size());
  size_t a = 0, b = 0, c = 0;
  cudaError_t e = cudaSuccess;
  for (size_t k = 0; k < ws.size() && e == cudaSuccess; ++k) {
    io[k] = a;
    to[k] = b;
    so[k] = c;
    e = cudaMemcpyAsync(d_insts_ + a, ws[k].insts.data(), sizeof(BatchInst<T>) * ws[k].insts.size(),
                        cudaMemcpyHostToDevice, stream_);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(d_tiles_ + b, ws[k].tiles.data(), sizeof(BatchTile) * ws[k].tiles.size(),
                          cudaMemcpyHostToDevice, stream_);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(d_items_ + c, ws[k].step_items.data(),
                          sizeof(long long) * ws[k].step_items.size(), cudaMemcpyHostToDevice, stream_);
    a += ws[k].insts.size();
    b += ws[k].tiles.size();
    c += ws[k].step_items.size();
  }
  if (e == cudaSuccess) e = cudaStreamSynchronize(stream_);
  if (e != cudaSuccess) return LE2D_ECUDA;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  e = cudaStreamBeginCapture(stream_, cudaStreamCaptureModeThreadLocal);
  if (e != cudaSuccess) return LE2D_ECUDA;
  for (size_t k = 0; k < ws.size() && rc == LE2D_OK; ++k) rc = launch_window(ws[k], io[k], to[k], so[k], to[k], k);
  cudaError_t e2 = cudaStreamEndCapture(stream_, &graph);
  if (rc != LE2D_OK || e2 != cudaSuccess) {
    if (graph) cudaGraphDestroy(graph);
    return LE2D_ECUDA;
  }
  e = cudaGraphInstantiate(&exec, graph, 0);
  cudaGraphDestroy(graph);
  if (e != cudaSuccess) return LE2D_ECUDA;
  e = cudaEventRecord(ev_[0], stream_);
  if (e == cudaSuccess) e = cudaGraphLaunch(exec, stream_);
  if (e == cudaSuccess) e = cudaEventRecord(ev_[1], stream_);
  if (e == cudaSuccess) e = cudaStreamSynchronize(stream_);
  float t = 0.0f;
  if (e == cudaSuccess) e = cudaEventElapsedTime(&t, ev_[0], ev_[1]);
  cudaGraphExecDestroy(exec);
  if (e != cudaSuccess) return LE2D_ECUDA;
  if (ms) *ms = t;
  std::vector<BatchCtl> ctl(ws.size());
  e = cudaMemcpy(ctl.data(), d_ctl_, sizeof(BatchCtl) * ws.size(), cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) return LE2D_ECUDA;
  // failures: a launch that ended early fails its instances and every later window's
  // (their states are not advanced consistently); otherwise only the marked instances
  bool aborted = false, any_failed = false;
  for (size_t k = 0; k < ws.size(); ++k) {
    if (ctl[k].status != 0) aborted = true;
    if (aborted)
      for (int id : ws[k].inst_ids) insts_[id].failed = true;
    if (ctl[k].failed != 0) any_failed = true;
  }
  if (any_failed) {
    std::vector<int> ids;
    for (int id = 0; id < (int)insts_.size(); ++id)
      if (insts_[id].live) ids.push_back(id);
    if (read_failures(ids) != LE2D_OK) return LE2D_ECUDA;
  }
  bool failed = false;
  for (const Window& w : ws)
    for (size_t k = 0; k < w.inst_ids.size(); ++k) {
      Inst& in = insts_[w.inst_ids[k]];
      if (in.failed) {
        failed = true;
        continue;
      }
      in.done_steps += w.inst_steps[k];
      in.cur ^= w.inst_items[k] & 1;
      node_updates_ += (long long)in.p.nx * in.p.ny * w.inst_steps[k];
    }
  return failed ? LE2D_ETIMEOUT : LE2D_OK;
}

template <typename T>
bool Engine<T>::finished(int id) const {
  return id >= 0 && id < (int)insts_.size() && insts_[id].done_steps >= insts_[id].p.steps;
}

template <typename T>
bool Engine<T>::failed(int id) const {
  return id >= 0 && id < (int)insts_.size() && insts_[id].failed;
}

template <typename T>
int Engine<T>::harvest_fields(int id, T* out) {
  if (id < 0 || id >= (int)insts_.size() || !out) return LE2D_EINVAL;
  const Inst& in = insts_[id];
  if (!in.live || in.failed || !finished(id)) return in.failed ? LE2D_ETIMEOUT : LE2D_ESTATE;
  if (!in.unpacked) return fields(id, out);  // no window ran (zero steps)
  cudaError_t e = cudaMemcpyAsync(out, in.buf[in.cur ^ 1], sizeof(T) * 5 * (size_t)in.p.nx * in.p.ny,
                                  cudaMemcpyDeviceToHost, copy_);
  if (e == cudaSuccess) e = cudaStreamSynchronize(copy_);
  return e == cudaSuccess ? LE2D_OK : LE2D_ECUDA;
}

template <typename T>
int Engine<T>::harvest_receivers(int id, T* out, int* nsamples) {
  if (id < 0 || id >= (int)insts_.size()) return LE2D_EINVAL;
  const Inst& in = insts_[id];
  if (!in.live || in.failed) return in.failed ? LE2D_ETIMEOUT : LE2D_ESTATE;
  const int have = in.trace ? (int)std::min<long long>(in.nsamples, in.done_steps / in.p.receiver_every) : 0;
  if (nsamples) *nsamples = have;
  if (!out || have == 0) return LE2D_OK;
  cudaError_t e = cudaMemcpy2DAsync(out, sizeof(T) * in.p.nx, in.trace, sizeof(T) * in.pitch,
                                    sizeof(T) * in.p.nx, 2 * (size_t)have, cudaMemcpyDeviceToHost, copy_);
  if (e == cudaSuccess) e = cudaStreamSynchronize(copy_);
  return e == cudaSuccess ? LE2D_OK : LE2D_ECUDA;
}

template <typename T>
int Engine<T>::fields(int id, T* out) {
  if (id < 0 || id >= (int)insts_.size() || !out) return LE2D_EINVAL;
  const Inst& in = insts_[id];
  if (!in.live) return LE2D_ESTATE;
  if (in.failed) return LE2D_ETIMEOUT;
  const int cur = in.cur;
  cudaError_t e = launch_unpack<T>(in.buf[cur], in.buf[cur ^ 1], in.p.nx, in.p.ny, in.pitch,
                                   in.plane, in.p.stype == ST_AOS, stream_);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(out, in.buf[cur ^ 1], sizeof(T) * 5 * (size_t)in.p.nx * in.p.ny,
                        cudaMemcpyDeviceToHost, stream_);
  if (e == cudaSuccess) e = cudaStreamSynchronize(stream_);
  return e == cudaSuccess ? LE2D_OK : LE2D_ECUDA;
}

template <typename T>
int Engine<T>::receivers(int id, T* out, int* nsamples) {
  if (id < 0 || id >= (int)insts_.size()) return LE2D_EINVAL;
  const Inst& in = insts_[id];
  if (!in.live) return LE2D_ESTATE;
  if (in.failed) return LE2D_ETIMEOUT;
  const int have = in.trace ? (int)std::min<long long>(in.nsamples, in.done_steps / in.p.receiver_every) : 0;
  if (nsamples) *nsamples = have;
  if (!out || have == 0) return LE2D_OK;
  cudaError_t e = cudaMemcpy2DAsync(out, sizeof(T) * in.p.nx, in.trace, sizeof(T) * in.pitch,
                                    sizeof(T) * in.p.nx, 2 * (size_t)have, cudaMemcpyDeviceToHost,
                                    stream_);
  if (e == cudaSuccess) e = cudaStreamSynchronize(stream_);
  return e == cudaSuccess ? LE2D_OK : LE2D_ECUDA;
}

template <typename T>
int Engine<T>::diagnostics(int id, le2d_diag_t* out) {
  if (id < 0 || id >= (int)insts_.size() || !out || !d_diag_) return LE2D_EINVAL;
  const Inst& in = insts_[id];
  if (!in.live) return LE2D_ESTATE;
  if (in.failed) return LE2D_ETIMEOUT;
  const double rho = in.p.rho, c1 = in.p.c1, c2 = in.p.c2;
  const double mu = rho * c2 * c2, la = rho * c1 * c1 - 2.0 * mu;
  double h[11];
  cudaError_t e = cudaMemsetAsync(d_diag_, 0, 11 * sizeof(double), stream_);
  if (e == cudaSuccess)
    e = launch_diag<T>(in.buf[in.cur], in.p.nx, in.p.ny, in.pitch, in.plane, rho,
                       (la + 2.0 * mu) / (8.0 * mu * (la + mu)), -2.0 * la / (8.0 * mu * (la + mu)),
                       1.0 / (2.0 * mu), d_diag_, stream_);
  if (e == cudaSuccess) e = cudaMemcpyAsync(h, d_diag_, sizeof(h), cudaMemcpyDeviceToHost, stream_);
  if (e == cudaSuccess) e = cudaStreamSynchronize(stream_);
  if (e != cudaSuccess) return LE2D_ECUDA;
  out->energy = h[0] * (double)in.p.hx * (double)in.p.hy;
  for (int k = 0; k < 5; ++k) {
    out->sumsq[k] = h[1 + k];
    out->maxabs[k] = h[6 + k];
  }
  return LE2D_OK;
}

template <typename T>
void Engine<T>::release(int id) {
  if (id < 0 || id >= (int)insts_.size()) return;
  Inst& in = insts_[id];
  if (!in.live) return;
  arena_->free(in.state_off);
  if (in.trace) arena_->free(in.trace_off);
  in.live = false;
  in.buf[0] = in.buf[1] = in.trace = nullptr;
}

template class Engine<real>;
template StepConsts<real> problem_consts<real>(const le2d_problem&);
template int batch_autotune<real>(int, int, BatchTuned*);

}  // namespace le2d

// ---------------------------------------------------------------- C API

struct le2d_batch {
  le2d::Engine<real>* eng;
};

extern "C" {

le2d_batch* le2d_batch_create(size_t device_budget_bytes) {
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) {
    cudaGetLastError();
    fprintf(stderr, "le2d: le2d_batch_create: no CUDA device\n");
    return nullptr;
  }
  auto* e = new le2d::Engine<real>(device_budget_bytes);
  if (!e->ok()) {
    fprintf(stderr, "le2d: le2d_batch_create: device setup failed\n");
    delete e;
    return nullptr;
  }
  return new le2d_batch{e};
}

void le2d_batch_destroy(le2d_batch* b) {
  if (!b) return;
  delete b->eng;
  delete b;
}

int le2d_batch_add(le2d_batch* b, const le2d_problem* p, const real* init, int ndisks,
                   const real* disks) {
  if (!b || !p) return -LE2D_EINVAL;
  return b->eng->add(*p, init, ndisks, disks);
}

int le2d_batch_run(le2d_batch* b, int window_steps, float* device_ms) {
  if (!b) return LE2D_EINVAL;
  const int rc = b->eng->run_all(window_steps, device_ms);
  if (rc) fprintf(stderr, "le2d: le2d_batch_run: %s\n", le2d_strerror(rc));
  return rc;
}

int le2d_batch_count(const le2d_batch* b) { return b ? b->eng->count() : 0; }

int le2d_batch_fields(le2d_batch* b, int id, real* out) {
  return b ? b->eng->fields(id, out) : LE2D_EINVAL;
}

int le2d_batch_receivers(le2d_batch* b, int id, real* out, int* nsamples) {
  return b ? b->eng->receivers(id, out, nsamples) : LE2D_EINVAL;
}

int le2d_batch_diagnostics(le2d_batch* b, int id, le2d_diag_t* out) {
  return b ? b->eng->diagnostics(id, out) : LE2D_EINVAL;
}

int le2d_batch_autotune(int nx, int ny, int* out, double* nu_per_s) {
  if (nx < 3 || ny < 3) return LE2D_EINVAL;
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) {
    cudaGetLastError();
    return LE2D_ENODEV;
  }
  le2d::BatchTuned t;
  const int rc = le2d::batch_autotune<real>(nx, ny, &t);
  if (rc) return rc;
  if (out) {
    out[0] = t.seg_len;
    out[1] = t.depth;
  }
  if (nu_per_s) *nu_per_s = t.nu_s;
  return LE2D_OK;
}

int le2d_batch_autotune_reset(void) {
  le2d::batch_tune_reset();
  return LE2D_OK;
}

int le2d_batch_set_wait_limit(le2d_batch* b, unsigned long long ns) {
  if (!b || ns == 0) return LE2D_EINVAL;
  b->eng->set_wait_ns(ns);
  return LE2D_OK;
}

}  // extern "C"
