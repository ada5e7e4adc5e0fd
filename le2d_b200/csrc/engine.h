// Host side of batched and served solves: a device arena for instance states, the
// per-window work lists of the persistent kernel (batch.cu), and result read-back.
// Used by le2d_batch_* (all instances known up front, windows captured in one CUDA
// graph) and by the serving loop (instances join and leave between windows).
#pragma once

#include <cuda_runtime.h>

#include <cstddef>
#include <map>
#include <vector>

#include "le2d.h"
#include "le2d_kernels.h"

namespace le2d {

// First-fit allocator over one cudaMalloc'd block; offsets are 256-byte aligned.
class Arena {
 public:
  explicit Arena(size_t capacity);
  ~Arena();
  bool ok() const { return base_ != nullptr; }
  // Returns an offset or SIZE_MAX when `bytes` does not fit.
  size_t alloc(size_t bytes);
  void free(size_t off);
  size_t capacity() const { return cap_; }
  size_t used() const { return used_; }
  char* base() const { return base_; }

 private:
  char* base_ = nullptr;
  size_t cap_ = 0, used_ = 0;
  std::map<size_t, size_t> free_;  // offset -> size
  std::map<size_t, size_t> live_;  // offset -> size
};

template <typename T>
class Engine {
 public:
  struct Inst {
    le2d_problem p;
    long long pitch = 0, plane = 0;
    size_t state_off = SIZE_MAX, trace_off = SIZE_MAX;
    T* buf[2] = {nullptr, nullptr};
    T* trace = nullptr;
    int nsamples = 0;
    long long done_steps = 0;
    int cur = 0;    // buffer holding the current state
    int depth = 1;  // steps per work item of the batched kernel
    StepConsts<T> c;
    int nstrips = 0, nsegs = 0, seg_len = 0;
    bool live = false;
    int* fail = nullptr;     // failure word on the device (in the instance's arena block)
    bool failed = false;     // a dependency wait of one of its tiles gave up: no results
    bool prologue = false;   // initial condition still to be applied (add_async)
    bool has_init = false;   //   from the host state uploaded into buf[1]
    std::vector<T> disks;    //   or from these disks (4 values each)
    bool unpacked = false;   // final fields unpacked into buf[cur ^ 1] after its last window
  };

  explicit Engine(size_t budget_bytes);
  ~Engine();
  bool ok() const { return arena_ && arena_->ok() && stream_ != nullptr; }
  cudaStream_t stream() const { return stream_; }

  // Device bytes an instance of this problem holds (states + receiver samples).
  static size_t footprint(const le2d_problem& p);
  // Validates, allocates and initialises an instance; returns its id or -LE2D_E*.
  int add(const le2d_problem& p, const T* init, int ndisks, const T* disks);
  // The same, for use while a window is in flight: allocates the instance and copies the
  // host initial state `init` into its second buffer on the copy stream (the call returns
  // once `init` has been read); the initial condition is applied on the step stream just
  // before the next window, so no kernel competes with the window for the SMs.
  int add_async(const le2d_problem& p, const T* init, int ndisks, const T* disks);
  // One window: every live instance with steps left advances by min(left, window) steps
  // in one persistent launch (not captured).  begin_window() applies pending initial
  // conditions, launches and returns; after the launch it also queues, on the step
  // stream, the unpacking of the final fields of the instances the window finishes.
  // end_window() waits for it: LE2D_OK (instances whose dependency wait gave up are
  // marked failed()), LE2D_ETIMEOUT (a wait inside a warp pair gave up: every instance
  // of the window failed) or LE2D_ECUDA.
  int begin_window(int window);
  int end_window();
  bool in_flight() const { return in_flight_; }
  // begin_window + end_window.
  int run_window(int window);
  // Runs every live instance to completion: all windows captured in one CUDA graph.
  // LE2D_ETIMEOUT if an instance failed (the others' results are valid).
  int run_all(int window, float* ms);
  int fields(int id, T* out);
  int receivers(int id, T* out, int* nsamples);
  // Results of an instance finished by an earlier window, read on the copy stream, so
  // they overlap a window in flight (fields: unpacked after the finishing window).
  int harvest_fields(int id, T* out);
  int harvest_receivers(int id, T* out, int* nsamples);
  int diagnostics(int id, le2d_diag_t* out);
  // Releases the instance's device memory (its results must have been read).
  void release(int id);
  bool finished(int id) const;
  bool failed(int id) const;
  int count() const { return (int)insts_.size(); }
  const Inst& inst(int id) const { return insts_[id]; }
  void set_wait_ns(unsigned long long ns) { wait_ns_ = ns; }
  // Tile height and steps per work item for instances added afterwards (the autotuner's
  // trials); otherwise they come from the autotuner's table for the instance's size class,
  // or the defaults (64 rows, batch_depth<T>()).
  int set_seg_len(int rows);
  int set_depth(int depth);
  // Whether instances added afterwards take their tiles from the autotuner's table (default)
  // or the defaults.  The serving loop uses the defaults: the table is tuned for throughput
  // on a full batch, and its taller tiles lengthen each small instance's chain of steps
  // (measured: untuned p50 latency 0.22 s against 0.39 s at 10 requests/s, and 46 against
  // 43 solves/s at 200).
  void set_use_tuned(bool on) { use_tuned_ = on; }
  size_t arena_used() const { return arena_ ? arena_->used() : 0; }
  size_t arena_capacity() const { return arena_ ? arena_->capacity() : 0; }
  long long node_updates() const { return node_updates_; }

 private:
  struct Window {
    std::vector<BatchInst<T>> insts;
    std::vector<BatchTile> tiles;
    std::vector<long long> step_items;  // size steps+1
    std::vector<int> inst_ids;
    std::vector<int> inst_steps;  // time steps of each instance in the window
    std::vector<int> inst_items;  // work-item steps of each instance (ceil(steps / depth))
    int steps = 0;                // work-item steps of the window
  };
  // done_steps / cur: each instance's steps so far and current buffer before the window.
  Window plan_window(int window, const std::vector<long long>& done_steps,
                     const std::vector<int>& cur) const;
  int ensure_scratch(size_t insts, size_t tiles, size_t items, size_t done, size_t ctls);
  int launch_window(const Window& w, size_t inst_off, size_t tile_off, size_t item_off,
                    size_t done_off, size_t ctl_off);

  int apply_prologues();  // pending initial conditions, on the step stream
  int alloc_instance(const le2d_problem& p, Inst& in);
  int read_failures(const std::vector<int>& ids);

  Arena* arena_ = nullptr;
  cudaStream_t stream_ = nullptr;
  cudaStream_t copy_ = nullptr;  // uploads and read-backs beside a window
  Window win_;                   // the window in flight
  bool in_flight_ = false;
  std::vector<Inst> insts_;
  unsigned long long wait_ns_ = 2000000000ULL;
  int stall_tile_ = -1;  // test hook from LE2D_TEST_STALL_TILE (see launch_batch): in the
                         // engine's first window only
  int seg_len_ = 64;
  bool seg_set_ = false;
  int depth_set_ = 0;
  bool use_tuned_ = true;
  int resident_blocks_ = 0;
  long long node_updates_ = 0;
  // device scratch of the persistent launches (work lists, counters)
  BatchInst<T>* d_insts_ = nullptr;
  BatchTile* d_tiles_ = nullptr;
  long long* d_items_ = nullptr;
  int* d_done_ = nullptr;
  BatchCtl* d_ctl_ = nullptr;
  size_t cap_insts_ = 0, cap_tiles_ = 0, cap_items_ = 0, cap_done_ = 0, cap_ctl_ = 0;
  double* d_diag_ = nullptr;
  cudaEvent_t ev_[2] = {nullptr, nullptr};
};

// Constants of one problem's step (same derivation as the single-solve path).
template <typename T>
StepConsts<T> problem_consts(const le2d_problem& p);

// Batched-path autotuner (per size class: nx, ny rounded up to powers of two): the fastest
// tile height and steps per work item measured on copies of a scratch problem.
struct BatchTuned {
  int seg_len = 0, depth = 0;
  double nu_s = 0.0;
};
template <typename T>
int batch_autotune(int nx, int ny, BatchTuned* out);
bool batch_tuned(int nx, int ny, BatchTuned* out);  // table lookup
void batch_tune_reset();

}  // namespace le2d
