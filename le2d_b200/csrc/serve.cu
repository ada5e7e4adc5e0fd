// Serving loop: continuous batching of forward-modelling solves on one GPU.
//
// One worker thread owns an Engine (device arena + persistent batched kernel).
// Clients call le2d_server_submit from any thread; the request (problem, initial
// condition) is copied into a ticket and queued.  The worker repeats:
//   1. admit queued requests, in arrival order, while the engine's arena can hold
//      their states (the HBM budget) and fewer than max_active run; their initial
//      states go to the device on a copy stream, beside the window in flight;
//   2. wait for the window in flight, if any;
//   3. launch the next window: every admitted solve with steps left advances by up to
//      window_steps steps in one persistent launch (solves of different sizes and
//      materials share it); the final fields of the solves it finishes are unpacked
//      right after it;
//   4. while that window runs, read back the results (final fields or receiver traces)
//      of the solves the previous window finished, on the copy stream, free their
//      device memory and wake the waiters.
// So requests that arrive while others are on the GPU join at the next window, their
// work overlaps with the others', and uploads and read-backs overlap the windows.  A
// solve whose tiles' dependency wait gave up fails alone (LE2D_ETIMEOUT); a launch that
// ended early fails the solves it carried.
#include <chrono>
#include <condition_variable>
#include <cstdio>
#include <cstring>
#include <deque>
#include <memory>
#include <mutex>
#include <thread>
#include <unordered_map>
#include <vector>

#include "engine.h"

namespace {

using T = real;

double now_s() {
  using namespace std::chrono;
  return duration<double>(steady_clock::now().time_since_epoch()).count();
}

struct Ticket {
  long long id = 0;
  le2d_problem p;
  std::vector<T> init;
  std::vector<T> disks;
  int want = LE2D_WANT_FIELDS;
  int status = 0;  // 0 pending, 1 done, -err failed
  int engine_id = -1;
  double t_submit = 0, t_admit = 0, t_done = 0;
  std::vector<T> result;
  int nsamples = 0;
};

}  // namespace

struct le2d_server {
  std::unique_ptr<le2d::Engine<T>> eng;
  int window = 100;
  int max_active = 1024;
  std::mutex mu;
  std::condition_variable cv_work, cv_done;
  std::deque<long long> queue;
  std::unordered_map<long long, std::shared_ptr<Ticket>> tickets;
  std::vector<std::shared_ptr<Ticket>> active;
  long long next_id = 1;
  bool stop = false;
  le2d_server_stats_t st{};
  std::thread worker;

  void finish(const std::shared_ptr<Ticket>& t, int status) {
    t->status = status;
    t->t_done = now_s();
    if (status == 1)
      ++st.completed;
    else
      ++st.failed;
  }

  void run() {
    std::unique_lock<std::mutex> lk(mu);
    double t_launch = 0.0;
    long long nu_launch = 0;
    while (true) {
      // 1. admission against the arena (HBM budget); the engine calls run unlocked
      std::vector<std::shared_ptr<Ticket>> cand;
      while (!stop && !queue.empty() && (int)(active.size() + cand.size()) < max_active) {
        auto it = tickets.find(queue.front());
        queue.pop_front();
        if (it != tickets.end()) cand.push_back(it->second);
      }
      const bool busy = !active.empty() || eng->in_flight();
      lk.unlock();
      std::vector<std::pair<std::shared_ptr<Ticket>, int>> added;  // ticket, engine id or -error
      size_t k = 0;
      for (; k < cand.size(); ++k) {
        const auto& t = cand[k];
        const int id = eng->add_async(t->p, t->init.empty() ? nullptr : t->init.data(),
                                      (int)(t->disks.size() / 4), t->disks.empty() ? nullptr : t->disks.data());
        if (id == -LE2D_EBUDGET && (busy || !added.empty())) break;  // wait for memory to free up
        added.push_back({t, id});
      }
      lk.lock();
      for (size_t j = cand.size(); j > k; --j) queue.push_front(cand[j - 1]->id);
      const double t_adm = now_s();
      for (auto& a : added) {
        if (a.second < 0) {
          finish(a.first, a.second);
          continue;
        }
        a.first->engine_id = a.second;
        a.first->t_admit = t_adm;
        a.first->init.clear();
        a.first->init.shrink_to_fit();
        active.push_back(a.first);
        ++st.admitted;
      }
      if (!added.empty()) cv_done.notify_all();
      if (stop) break;
      if (active.empty() && !eng->in_flight()) {
        cv_work.wait(lk, [&] { return stop || !queue.empty(); });
        continue;
      }
      lk.unlock();
      // 2. the window in flight
      int rc = LE2D_OK;
      if (eng->in_flight()) {
        rc = eng->end_window();
        const double t1 = now_s();
        std::lock_guard<std::mutex> g(mu);
        st.device_busy_s += t1 - t_launch;
        st.node_updates += eng->node_updates() - nu_launch;
        ++st.windows;
      }
      // 3. the next window
      if (rc != LE2D_ECUDA) {
        t_launch = now_s();
        nu_launch = eng->node_updates();
        rc = eng->begin_window(window);
        if (rc == LE2D_ETIMEOUT) rc = LE2D_OK;  // per-solve failures are read below
      }
      // 4. results of the solves that are done, read beside the new window
      std::vector<std::pair<std::shared_ptr<Ticket>, int>> done;  // ticket, final status
      for (auto& t : active) {
        const int id = t->engine_id;
        int status = 0;
        if (rc == LE2D_ECUDA) {
          status = -LE2D_ECUDA;
        } else if (eng->failed(id)) {
          status = -LE2D_ETIMEOUT;
        } else if (eng->finished(id)) {
          int r2 = LE2D_OK;
          if (t->want == LE2D_WANT_RECEIVERS) {
            int n = 0;
            r2 = eng->harvest_receivers(id, nullptr, &n);
            t->result.resize((size_t)n * 2 * t->p.nx);
            t->nsamples = n;
            if (r2 == LE2D_OK && n > 0) r2 = eng->harvest_receivers(id, t->result.data(), &n);
          } else {
            t->result.resize((size_t)5 * t->p.nx * t->p.ny);
            r2 = eng->harvest_fields(id, t->result.data());
          }
          status = r2 == LE2D_OK ? 1 : -r2;
        }
        if (status != 0) {
          eng->release(id);
          done.push_back({t, status});
        }
      }
      lk.lock();
      if (!done.empty()) {
        std::vector<std::shared_ptr<Ticket>> keep;
        for (auto& t : active) {
          bool fin = false;
          for (auto& d : done) fin = fin || d.first == t;
          if (!fin) keep.push_back(t);
        }
        for (auto& d : done) finish(d.first, d.second);
        active.swap(keep);
        cv_done.notify_all();
      }
    }
    lk.unlock();
    if (eng->in_flight()) eng->end_window();
    lk.lock();
    for (auto& t : active) eng->release(t->engine_id);
    active.clear();
  }
};

extern "C" {

double le2d_now(void) { return now_s(); }

le2d_server* le2d_server_create(size_t device_budget_bytes, int window_steps, int max_active) {
  if (window_steps < 1 || max_active < 1) return nullptr;
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) {
    cudaGetLastError();
    fprintf(stderr, "le2d: le2d_server_create: no CUDA device\n");
    return nullptr;
  }
  auto* s = new le2d_server();
  s->eng.reset(new le2d::Engine<T>(device_budget_bytes));
  if (!s->eng->ok()) {
    fprintf(stderr, "le2d: le2d_server_create: device setup failed\n");
    delete s;
    return nullptr;
  }
  s->eng->set_use_tuned(false);  // default tiles: shorter chains per small solve (engine.h)
  s->window = window_steps;
  s->max_active = max_active;
  int dev = 0;
  cudaGetDevice(&dev);
  s->worker = std::thread([s, dev] {
    cudaSetDevice(dev);
    s->run();
  });
  return s;
}

void le2d_server_destroy(le2d_server* s) {
  if (!s) return;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    s->stop = true;
  }
  s->cv_work.notify_all();
  if (s->worker.joinable()) s->worker.join();
  delete s;
}

long long le2d_server_submit(le2d_server* s, const le2d_problem* p, const real* init, int ndisks,
                             const real* disks, int want) {
  if (!s || !p || ndisks < 0 || (ndisks > 0 && !disks)) return -LE2D_EINVAL;
  if (want != LE2D_WANT_FIELDS && want != LE2D_WANT_RECEIVERS) return -LE2D_EINVAL;
  if (want == LE2D_WANT_RECEIVERS && (p->receiver_row < 0 || p->receiver_every < 1))
    return -LE2D_EINVAL;
  if (p->nx < 3 || p->ny < 3 || p->steps < 0) return -LE2D_EINVAL;
  if (le2d::Engine<T>::footprint(*p) > s->eng->arena_capacity()) return -LE2D_EBUDGET;
  auto t = std::make_shared<Ticket>();
  t->p = *p;
  if (init) t->init.assign(init, init + (size_t)5 * p->nx * p->ny);
  if (ndisks > 0) t->disks.assign(disks, disks + 4 * (size_t)ndisks);
  t->want = want;
  t->t_submit = now_s();
  {
    std::lock_guard<std::mutex> lk(s->mu);
    t->id = s->next_id++;
    s->tickets[t->id] = t;
    s->queue.push_back(t->id);
    ++s->st.submitted;
  }
  s->cv_work.notify_all();
  return t->id;
}

int le2d_server_poll(le2d_server* s, long long ticket) {
  if (!s) return -LE2D_EINVAL;
  std::lock_guard<std::mutex> lk(s->mu);
  auto it = s->tickets.find(ticket);
  if (it == s->tickets.end()) return -LE2D_EINVAL;
  return it->second->status;
}

int le2d_server_wait(le2d_server* s, long long ticket, double timeout_s) {
  if (!s) return LE2D_EINVAL;
  std::unique_lock<std::mutex> lk(s->mu);
  auto it = s->tickets.find(ticket);
  if (it == s->tickets.end()) return LE2D_EINVAL;
  std::shared_ptr<Ticket> t = it->second;
  auto ready = [&] { return t->status != 0; };
  if (timeout_s < 0)
    s->cv_done.wait(lk, ready);
  else if (!s->cv_done.wait_for(lk, std::chrono::duration<double>(timeout_s), ready))
    return LE2D_ETIMEOUT;
  return t->status == 1 ? LE2D_OK : -t->status;
}

int le2d_server_result(le2d_server* s, long long ticket, real* out, size_t out_elems, int* nsamples) {
  if (!s) return LE2D_EINVAL;
  std::lock_guard<std::mutex> lk(s->mu);
  auto it = s->tickets.find(ticket);
  if (it == s->tickets.end()) return LE2D_EINVAL;
  const Ticket& t = *it->second;
  if (t.status == 0) return LE2D_ESTATE;
  if (t.status < 0) return -t.status;
  if (nsamples) *nsamples = t.nsamples;
  if (!out) return LE2D_OK;
  if (out_elems < t.result.size()) return LE2D_EINVAL;
  memcpy(out, t.result.data(), sizeof(T) * t.result.size());
  return LE2D_OK;
}

int le2d_server_times(le2d_server* s, long long ticket, double* t_submit, double* t_admit,
                      double* t_done) {
  if (!s) return LE2D_EINVAL;
  std::lock_guard<std::mutex> lk(s->mu);
  auto it = s->tickets.find(ticket);
  if (it == s->tickets.end()) return LE2D_EINVAL;
  if (t_submit) *t_submit = it->second->t_submit;
  if (t_admit) *t_admit = it->second->t_admit;
  if (t_done) *t_done = it->second->t_done;
  return LE2D_OK;
}

int le2d_server_release(le2d_server* s, long long ticket) {
  if (!s) return LE2D_EINVAL;
  std::lock_guard<std::mutex> lk(s->mu);
  auto it = s->tickets.find(ticket);
  if (it == s->tickets.end()) return LE2D_EINVAL;
  if (it->second->status == 0) return LE2D_ESTATE;
  s->tickets.erase(it);
  return LE2D_OK;
}

int le2d_server_stats(le2d_server* s, le2d_server_stats_t* out) {
  if (!s || !out) return LE2D_EINVAL;
  std::lock_guard<std::mutex> lk(s->mu);
  *out = s->st;
  out->arena_used = s->eng->arena_used();
  out->arena_capacity = s->eng->arena_capacity();
  out->active = (int)s->active.size();
  out->queued = (int)s->queue.size();
  return LE2D_OK;
}

}  // extern "C"
