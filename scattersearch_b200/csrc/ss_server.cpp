// Serving loop of the C ABI (ss_server_* in include/scattersearch.h).
//
// The reference serves online queries with a generator thread, a
// mutex-guarded deque and one consumer that searches one query at a time
// (tests/online_parallel_search.cpp:91-160).  Here a dispatcher thread owns
// a few launch slots, each a CUDA stream with fixed device and pinned host
// buffers for max_batch requests.  Whenever a slot is free and requests are
// pending, it launches all of them (up to max_batch, each with its own K and
// L) as one batched search on that slot's stream, followed by an event.  A
// completion thread polls the events of the slots in flight and marks each
// slot done as its event completes.  Polling costs up to one host core while
// batches are in flight; blocking event waits and host callbacks were both
// measured to wake up tens of milliseconds late now and then (p99 at 1k
// requests/s: 23 ms blocking against 1.35 ms polling).  Requests arriving while launches run wait only for the next
// free slot, and launches on different slots overlap on the device (each
// grid is sized to its own batch).  Every query's result is independent of
// its batch: the kernel keeps no state shared between queries.
//
// Requests live in a preallocated ring of max_pending entries indexed by
// ticket (query, K/L, arrival time, results): tickets are dense and
// dispatched in order, so the pending ones are exactly [next_dispatch,
// next_ticket) and submitting allocates nothing.  A ring entry is reused once
// its ticket has been collected by ss_server_wait.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <memory>
#include <mutex>
#include <thread>
#include <vector>

#include "scattersearch.h"
#include "ss_internal.h"

namespace {

using Clock = std::chrono::steady_clock;

enum ReqState { kPending = 0, kRunning = 1, kDone = 2, kFailed = 3 };

enum : int { kFree = -1 };

struct Request {
  int K = 0, L = 0;
  Clock::time_point t_arrival;
  int state = kFree;
  double latency_us = 0.0;
};

struct Slot {
  cudaStream_t stream = nullptr;
  // device
  float *d_q = nullptr, *d_dists = nullptr;
  int32_t *d_K = nullptr, *d_L = nullptr, *d_status = nullptr;
  int64_t *d_off = nullptr;
  uint32_t *d_ids = nullptr, *d_counter = nullptr;
  // pinned host
  float *h_q = nullptr, *h_dists = nullptr;
  int32_t *h_K = nullptr, *h_L = nullptr, *h_status = nullptr;
  int64_t *h_off = nullptr;
  uint32_t *h_ids = nullptr;
  // in flight
  std::vector<uint64_t> tickets;
  bool busy = false;
  bool launch_failed = false;
  std::atomic<bool> done{false};
  Clock::time_point t_done;
  struct ss_server *owner = nullptr;
  // completion: the event recorded after a batch's result copies; armed
  // (under the server's poll_mu) while the completion thread watches it
  cudaEvent_t done_ev = nullptr;
  bool armed = false;
};

template <class T>
cudaError_t dev_alloc(T **p, size_t n) {
  return cudaMalloc(reinterpret_cast<void **>(p), std::max<size_t>(n, 1) * sizeof(T));
}
template <class T>
cudaError_t host_alloc(T **p, size_t n) {
  return cudaMallocHost(reinterpret_cast<void **>(p), std::max<size_t>(n, 1) * sizeof(T));
}

double pct(std::vector<double> v, double q) {
  if (v.empty()) return 0.0;
  const size_t k = std::min(v.size() - 1, (size_t)(q * (double)(v.size() - 1) + 0.5));
  std::nth_element(v.begin(), v.begin() + (long)k, v.end());
  return v[k];
}

}  // namespace

struct ss_server {
  ss_index *h = nullptr;
  int device = 0;
  uint32_t dim = 0;
  ss_server_config cfg{};
  std::vector<std::unique_ptr<Slot>> slots;

  std::mutex mu;
  std::condition_variable cv_work, cv_done;
  // request ring (max_pending entries), indexed by ticket % cap
  uint64_t cap = 0;
  std::vector<Request> ring;
  std::vector<float> ring_q;      // cap x dim
  std::vector<uint32_t> ring_ids; // cap x K_max
  std::vector<float> ring_d;      // cap x K_max
  uint64_t next_ticket = 0;       // next ticket to hand out
  uint64_t next_dispatch = 0;     // first ticket not yet launched
  uint64_t oldest = 0;            // first ticket not yet collected
  bool stop = false;
  std::thread dispatcher;
  // completion thread: polls the events of armed slots
  std::thread poller;
  std::mutex poll_mu;
  std::condition_variable poll_cv;
  int n_armed = 0;
  bool poll_quit = false;
  void poll_run();

  Request &req(uint64_t t) { return ring[t % cap]; }
  uint64_t pending() const { return next_ticket - next_dispatch; }

  // statistics
  uint64_t n_submitted = 0, n_completed = 0, n_failed = 0, n_batches = 0, n_batched = 0;
  std::vector<double> latencies;

  void run();
  void finish_slot(Slot &sl);
  bool launch_slot(Slot &sl, std::unique_lock<std::mutex> &lk);
  int submit_at(const float *query, int K, int L, Clock::time_point t_arrival, uint64_t *ticket);
  // Submits up to `count` requests at once (one lock, one wake-up); returns
  // how many went in before the ring filled (or a negative error status).
  int submit_many(const float *queries, const int32_t *Ks, const int32_t *Ls,
                  const Clock::time_point *t_arrival, uint32_t count, uint64_t *tickets);
  void free_slots();
};

namespace {

constexpr size_t kMaxLatencySamples = size_t(1) << 22;

}  // namespace

// Copies a finished slot's results to its requests (mu held).
void ss_server::finish_slot(Slot &sl) {
  const size_t kx = (size_t)cfg.K_max;
  for (size_t i = 0; i < sl.tickets.size(); ++i) {
    const uint64_t t = sl.tickets[i];
    Request &r = req(t);
    const bool ok = !sl.launch_failed && sl.h_status[i] == ssb::kStatusOk;
    if (ok) {
      std::memcpy(&ring_ids[(t % cap) * kx], sl.h_ids + sl.h_off[i], (size_t)r.K * 4);
      std::memcpy(&ring_d[(t % cap) * kx], sl.h_dists + sl.h_off[i], (size_t)r.K * 4);
    }
    r.latency_us = std::chrono::duration<double, std::micro>(sl.t_done - r.t_arrival).count();
    r.state = ok ? kDone : kFailed;
    if (ok) {
      ++n_completed;
      if (latencies.size() < kMaxLatencySamples) latencies.push_back(r.latency_us);
    } else {
      ++n_failed;
    }
  }
  sl.tickets.clear();
  sl.busy = false;
  sl.launch_failed = false;
  sl.done.store(false, std::memory_order_relaxed);
  cv_done.notify_all();
}

// Launches up to max_batch pending requests on a free slot (mu held on
// entry and exit).  Returns false if nothing was launched.
bool ss_server::launch_slot(Slot &sl, std::unique_lock<std::mutex> &lk) {
  if (pending() == 0) return false;
  const uint32_t nb = (uint32_t)std::min<uint64_t>(pending(), cfg.max_batch);
  const uint64_t t0 = next_dispatch;
  next_dispatch += nb;
  sl.tickets.resize(nb);
  int64_t off = 0;
  int L_max = 1;
  for (uint32_t i = 0; i < nb; ++i) {
    Request &r = req(t0 + i);
    sl.tickets[i] = t0 + i;
    sl.h_K[i] = r.K;
    sl.h_L[i] = r.L;
    sl.h_off[i] = off;
    off += r.K;
    L_max = std::max(L_max, r.L);
    r.state = kRunning;
  }
  sl.busy = true;
  sl.done.store(false, std::memory_order_relaxed);
  lk.unlock();
  // The ring entries of these tickets stay untouched until they are
  // collected, so their queries are copied without the lock.
  for (uint32_t i = 0; i < nb; ++i)
    std::memcpy(sl.h_q + (size_t)i * dim, &ring_q[((t0 + i) % cap) * dim],
                (size_t)dim * sizeof(float));
  // Enqueue: inputs up, search, results down, completion callback.
  bool ok = cudaMemcpyAsync(sl.d_q, sl.h_q, (size_t)nb * dim * sizeof(float),
                            cudaMemcpyHostToDevice, sl.stream) == cudaSuccess &&
            cudaMemcpyAsync(sl.d_K, sl.h_K, nb * sizeof(int32_t), cudaMemcpyHostToDevice,
                            sl.stream) == cudaSuccess &&
            cudaMemcpyAsync(sl.d_L, sl.h_L, nb * sizeof(int32_t), cudaMemcpyHostToDevice,
                            sl.stream) == cudaSuccess &&
            cudaMemcpyAsync(sl.d_off, sl.h_off, nb * sizeof(int64_t), cudaMemcpyHostToDevice,
                            sl.stream) == cudaSuccess;
  if (ok)
    ok = ssb::server_launch(h, sl.d_q, nb, sl.d_K, sl.d_L, sl.d_off, L_max, sl.d_ids, sl.d_dists,
                            sl.d_status, sl.d_counter, sl.stream) == SS_OK;
  if (ok)
    ok = cudaMemcpyAsync(sl.h_ids, sl.d_ids, (size_t)off * sizeof(uint32_t),
                         cudaMemcpyDeviceToHost, sl.stream) == cudaSuccess &&
         cudaMemcpyAsync(sl.h_dists, sl.d_dists, (size_t)off * sizeof(float),
                         cudaMemcpyDeviceToHost, sl.stream) == cudaSuccess &&
         cudaMemcpyAsync(sl.h_status, sl.d_status, nb * sizeof(int32_t),
                         cudaMemcpyDeviceToHost, sl.stream) == cudaSuccess;
  sl.launch_failed = !ok;
  if (cudaEventRecord(sl.done_ev, sl.stream) == cudaSuccess) {
    {
      std::lock_guard<std::mutex> pl(poll_mu);
      sl.armed = true;
      ++n_armed;
    }
    poll_cv.notify_one();
  } else {
    // nothing will signal this launch: complete the slot here (as failed)
    sl.launch_failed = true;
    sl.t_done = Clock::now();
    sl.done.store(true, std::memory_order_release);
  }
  lk.lock();
  ++n_batches;
  n_batched += nb;
  return true;
}

void ss_server::run() {
  cudaSetDevice(device);
  std::unique_lock<std::mutex> lk(mu);
  for (;;) {
    for (auto &sl : slots)
      if (sl->busy && sl->done.load(std::memory_order_acquire)) finish_slot(*sl);
    bool any_busy = false;
    for (auto &sl : slots) {
      if (!sl->busy && !stop) launch_slot(*sl, lk);
      any_busy = any_busy || sl->busy;
    }
    if (stop && !any_busy) break;
    cv_work.wait(lk, [&] {
      for (auto &sl : slots) {
        if (sl->busy && sl->done.load(std::memory_order_acquire)) return true;
        if (!sl->busy && pending() > 0 && !stop) return true;
      }
      if (stop) {
        for (auto &sl : slots)
          if (sl->busy) return false;
        return true;
      }
      return false;
    });
  }
}

int ss_server::submit_at(const float *query, int K, int L, Clock::time_point t_arrival,
                         uint64_t *ticket) {
  if (!query || !ticket) return ssb::index_error(h, SS_ERR_INVALID_ARGUMENT, "null query or ticket");
  if (K < 1 || K > L || K > cfg.K_max || L > cfg.L_max)
    return ssb::index_error(h, SS_ERR_INVALID_ARGUMENT,
                            "request needs 1 <= K <= L, K <= K_max and L <= L_max");
  {
    std::lock_guard<std::mutex> lk(mu);
    if (stop) return ssb::index_error(h, SS_ERR_INVALID_ARGUMENT, "server is stopping");
    if (next_ticket - oldest >= cap)
      return ssb::index_error(h, SS_ERR_BUSY, "request queue is full");
    const uint64_t t = next_ticket++;
    Request &r = req(t);
    std::memcpy(&ring_q[(t % cap) * dim], query, (size_t)dim * sizeof(float));
    r.K = K;
    r.L = L;
    r.t_arrival = t_arrival;
    r.state = kPending;
    ++n_submitted;
    *ticket = t + 1;  // tickets handed out start at 1
  }
  cv_work.notify_all();
  return SS_OK;
}

int ss_server::submit_many(const float *queries, const int32_t *Ks, const int32_t *Ls,
                           const Clock::time_point *t_arrival, uint32_t count,
                           uint64_t *tickets) {
  for (uint32_t i = 0; i < count; ++i)
    if (Ks[i] < 1 || Ks[i] > Ls[i] || Ks[i] > cfg.K_max || Ls[i] > cfg.L_max)
      return -ssb::index_error(h, SS_ERR_INVALID_ARGUMENT,
                               "request needs 1 <= K <= L, K <= K_max and L <= L_max");
  uint32_t n = 0;
  {
    std::lock_guard<std::mutex> lk(mu);
    if (stop) return -ssb::index_error(h, SS_ERR_INVALID_ARGUMENT, "server is stopping");
    for (; n < count && next_ticket - oldest < cap; ++n) {
      const uint64_t t = next_ticket++;
      Request &r = req(t);
      std::memcpy(&ring_q[(t % cap) * dim], queries + (size_t)n * dim, (size_t)dim * sizeof(float));
      r.K = Ks[n];
      r.L = Ls[n];
      r.t_arrival = t_arrival[n];
      r.state = kPending;
      ++n_submitted;
      tickets[n] = t + 1;  // tickets handed out start at 1
    }
  }
  if (n) cv_work.notify_all();
  return (int)n;
}

// Completion thread: while any slot is armed, checks each armed slot's event
// without blocking (cudaEventQuery) and yields between sweeps; sleeps on
// poll_cv while nothing is in flight.  A query that reports an error marks
// the batch failed.
void ss_server::poll_run() {
  cudaSetDevice(device);
  for (;;) {
    {
      std::unique_lock<std::mutex> pl(poll_mu);
      poll_cv.wait(pl, [this] { return n_armed > 0 || poll_quit; });
      if (n_armed == 0) return;  // quit with nothing in flight
    }
    bool any = false;
    for (auto &sl : slots) {
      {
        std::lock_guard<std::mutex> pl(poll_mu);
        if (!sl->armed) continue;
      }
      const cudaError_t e = cudaEventQuery(sl->done_ev);
      if (e == cudaErrorNotReady) continue;
      sl->t_done = Clock::now();
      if (e != cudaSuccess) sl->launch_failed = true;
      {
        std::lock_guard<std::mutex> pl(poll_mu);
        sl->armed = false;
        --n_armed;
      }
      sl->done.store(true, std::memory_order_release);
      any = true;
    }
    if (any) {
      { std::lock_guard<std::mutex> lk(mu); }
      cv_work.notify_all();
    } else {
      std::this_thread::yield();
    }
  }
}

void ss_server::free_slots() {
  if (poller.joinable()) {
    {
      std::lock_guard<std::mutex> pl(poll_mu);
      poll_quit = true;
    }
    poll_cv.notify_one();
    poller.join();
  }
  for (auto &sl : slots) {
    if (sl->done_ev) cudaEventDestroy(sl->done_ev);
    if (sl->stream) cudaStreamDestroy(sl->stream);
    cudaFree(sl->d_q);
    cudaFree(sl->d_dists);
    cudaFree(sl->d_K);
    cudaFree(sl->d_L);
    cudaFree(sl->d_status);
    cudaFree(sl->d_off);
    cudaFree(sl->d_ids);
    cudaFree(sl->d_counter);
    cudaFreeHost(sl->h_q);
    cudaFreeHost(sl->h_dists);
    cudaFreeHost(sl->h_K);
    cudaFreeHost(sl->h_L);
    cudaFreeHost(sl->h_status);
    cudaFreeHost(sl->h_off);
    cudaFreeHost(sl->h_ids);
  }
  slots.clear();
}

extern "C" {

int ss_server_create(ss_index *h, const ss_server_config *cfg, ss_server **out) {
  if (!out) return ssb::index_error(h, SS_ERR_INVALID_ARGUMENT, "null output");
  *out = nullptr;
  if (!ssb::index_ready(h)) {
    if (!h) return ssb::index_error(nullptr, SS_ERR_INVALID_ARGUMENT, "null index handle");
    return ssb::index_error(h, SS_ERR_NO_GRAPH, "no graph loaded");
  }
  ss_server_config c{};
  if (cfg) c = *cfg;
  if (c.max_batch == 0) c.max_batch = 256;
  if (c.max_inflight == 0) c.max_inflight = 4;
  if (c.max_pending == 0) c.max_pending = 1u << 14;
  if (c.K_max == 0) c.K_max = 100;
  if (c.L_max == 0) c.L_max = 512;
  if (c.memory_fraction <= 0.f) c.memory_fraction = 0.25f;
  if (c.max_batch > 4096 || c.max_inflight > 16 || c.max_pending > (1u << 24) || c.K_max < 1 ||
      c.L_max < c.K_max ||
      c.L_max > SS_MAX_L || c.memory_fraction > 1.f)
    return ssb::index_error(h, SS_ERR_INVALID_ARGUMENT, "server configuration out of range");

  auto s = std::make_unique<ss_server>();
  s->h = h;
  s->device = ssb::index_device(h);
  s->dim = ssb::index_dim(h);
  s->cfg = c;
  s->cap = c.max_pending;
  s->ring.resize(s->cap);
  s->ring_q.resize((size_t)s->cap * s->dim);
  s->ring_ids.resize((size_t)s->cap * (size_t)c.K_max);
  s->ring_d.resize((size_t)s->cap * (size_t)c.K_max);
  s->latencies.reserve(kMaxLatencySamples);
  int prev = 0;
  cudaGetDevice(&prev);
  cudaSetDevice(s->device);
  // Admission by device memory: as many slots as the budget holds, at most
  // max_inflight.
  const size_t B = c.max_batch, Kx = (size_t)c.K_max;
  const size_t per_slot = B * (s->dim * 4 + 4 + 4 + 8 + 4) + B * Kx * 8 + 64;
  size_t free_b = 0, total_b = 0;
  if (cudaMemGetInfo(&free_b, &total_b) != cudaSuccess) {
    cudaSetDevice(prev);
    return ssb::index_error(h, SS_ERR_CUDA, "cudaMemGetInfo failed");
  }
  const size_t budget = (size_t)((double)free_b * c.memory_fraction);
  const size_t n_slots = std::min<size_t>(c.max_inflight, budget / per_slot);
  if (n_slots < 1) {
    cudaSetDevice(prev);
    return ssb::index_error(h, SS_ERR_OUT_OF_MEMORY,
                            "free device memory does not hold one launch slot");
  }
  bool ok = true;
  for (size_t i = 0; i < n_slots && ok; ++i) {
    auto sl = std::make_unique<Slot>();
    sl->owner = s.get();
    ok = cudaStreamCreateWithFlags(&sl->stream, cudaStreamNonBlocking) == cudaSuccess &&
         cudaEventCreateWithFlags(&sl->done_ev, cudaEventDisableTiming) == cudaSuccess &&
         dev_alloc(&sl->d_q, B * s->dim) == cudaSuccess &&
         dev_alloc(&sl->d_K, B) == cudaSuccess && dev_alloc(&sl->d_L, B) == cudaSuccess &&
         dev_alloc(&sl->d_off, B) == cudaSuccess && dev_alloc(&sl->d_ids, B * Kx) == cudaSuccess &&
         dev_alloc(&sl->d_dists, B * Kx) == cudaSuccess &&
         dev_alloc(&sl->d_status, B) == cudaSuccess && dev_alloc(&sl->d_counter, 4) == cudaSuccess &&
         host_alloc(&sl->h_q, B * s->dim) == cudaSuccess &&
         host_alloc(&sl->h_K, B) == cudaSuccess && host_alloc(&sl->h_L, B) == cudaSuccess &&
         host_alloc(&sl->h_off, B) == cudaSuccess && host_alloc(&sl->h_ids, B * Kx) == cudaSuccess &&
         host_alloc(&sl->h_dists, B * Kx) == cudaSuccess &&
         host_alloc(&sl->h_status, B) == cudaSuccess;
    s->slots.push_back(std::move(sl));
  }
  if (!ok) {
    s->free_slots();
    cudaSetDevice(prev);
    return ssb::index_error(h, SS_ERR_OUT_OF_MEMORY, "launch slot allocation failed");
  }
  cudaSetDevice(prev);
  ss_server *raw = s.get();
  raw->poller = std::thread([raw] { raw->poll_run(); });
  raw->dispatcher = std::thread([raw] { raw->run(); });
  *out = s.release();
  return SS_OK;
}

int ss_server_submit(ss_server *s, const float *query, int K, int L, uint64_t *ticket) {
  if (!s) return ssb::index_error(nullptr, SS_ERR_INVALID_ARGUMENT, "null server");
  return s->submit_at(query, K, L, Clock::now(), ticket);
}

int ss_server_wait(ss_server *s, uint64_t ticket, int timeout_ms, uint32_t *ids, float *dists,
                   double *latency_us) {
  if (!s) return ssb::index_error(nullptr, SS_ERR_INVALID_ARGUMENT, "null server");
  std::unique_lock<std::mutex> lk(s->mu);
  const uint64_t t = ticket - 1;
  if (ticket == 0 || t < s->oldest || t >= s->next_ticket || s->req(t).state == kFree)
    return ssb::index_error(s->h, SS_ERR_INVALID_ARGUMENT, "unknown ticket");
  Request &r = s->req(t);
  auto ready = [&] { return r.state >= kDone; };
  if (timeout_ms < 0) {
    s->cv_done.wait(lk, ready);
  } else if (!s->cv_done.wait_for(lk, std::chrono::milliseconds(timeout_ms), ready)) {
    return ssb::index_error(s->h, SS_ERR_TIMEOUT, "request not finished within the timeout");
  }
  const bool ok = r.state == kDone;
  const size_t kx = (size_t)s->cfg.K_max;
  if (ok && ids) std::memcpy(ids, &s->ring_ids[(t % s->cap) * kx], (size_t)r.K * sizeof(uint32_t));
  if (ok && dists) std::memcpy(dists, &s->ring_d[(t % s->cap) * kx], (size_t)r.K * sizeof(float));
  if (latency_us) *latency_us = r.latency_us;
  r.state = kFree;
  while (s->oldest < s->next_ticket && s->req(s->oldest).state == kFree) ++s->oldest;
  if (!ok) return ssb::index_error(s->h, SS_ERR_SEARCH_LIMIT, "request failed on the device");
  return SS_OK;
}

int ss_server_replay(ss_server *s, const float *queries, uint32_t nq, const int32_t *Ks,
                     const int32_t *Ls, const double *arrival_us, uint32_t *ids, float *dists,
                     double *latency_us) {
  if (!s) return ssb::index_error(nullptr, SS_ERR_INVALID_ARGUMENT, "null server");
  if (nq == 0) return SS_OK;
  if (!queries || !Ks || !Ls || !arrival_us || !ids)
    return ssb::index_error(s->h, SS_ERR_INVALID_ARGUMENT, "null replay argument");
  std::vector<uint64_t> tickets(nq, 0);
  std::vector<int64_t> off(nq, 0);
  for (uint32_t i = 1; i < nq; ++i) off[i] = off[i - 1] + Ks[i - 1];
  std::atomic<int> gen_rc{SS_OK};
  // The generator sleeps until the next arrival time and then submits every
  // request that is due in one go (it never spins: a busy client thread
  // competes with the dispatcher for the host's cores); latency still runs
  // from each request's scheduled arrival, so a late wake-up counts against
  // the server.
  std::mutex sub_mu;
  std::condition_variable sub_cv;
  uint32_t submitted = 0;
  const Clock::time_point t0 = Clock::now();
  std::vector<Clock::time_point> t_arr(nq);
  for (uint32_t i = 0; i < nq; ++i)
    t_arr[i] = t0 + std::chrono::duration_cast<Clock::duration>(
                        std::chrono::duration<double, std::micro>(arrival_us[i]));
  std::thread gen([&] {
    uint32_t i = 0;
    while (i < nq) {
      if (Clock::now() < t_arr[i]) std::this_thread::sleep_until(t_arr[i]);
      const Clock::time_point now = Clock::now();
      uint32_t due = i + 1;
      while (due < nq && t_arr[due] <= now && due - i < 4096) ++due;
      const int n = s->submit_many(queries + (size_t)i * s->dim, Ks + i, Ls + i, t_arr.data() + i,
                                   due - i, tickets.data() + i);
      if (n < 0) {
        gen_rc.store(-n);
        std::lock_guard<std::mutex> lk(sub_mu);
        submitted = nq + 1;  // stopped early
      } else {
        i += (uint32_t)n;
        std::lock_guard<std::mutex> lk(sub_mu);
        submitted = i;
      }
      sub_cv.notify_one();
      if (n < 0) break;
      if (n == 0) std::this_thread::sleep_for(std::chrono::microseconds(50));  // ring full
    }
  });
  int rc = SS_OK;
  for (uint32_t i = 0; i < nq; ++i) {
    {
      std::unique_lock<std::mutex> lk(sub_mu);
      sub_cv.wait(lk, [&] { return submitted > i; });
      if (submitted == nq + 1 && tickets[i] == 0) break;
    }
    double lat = 0.0;
    const int w = ss_server_wait(s, tickets[i], -1, ids + off[i], dists ? dists + off[i] : nullptr,
                                 &lat);
    if (latency_us) latency_us[i] = lat;
    if (w != SS_OK && rc == SS_OK) rc = w;
  }
  gen.join();
  if (gen_rc.load() != SS_OK) return gen_rc.load();
  return rc;
}

int ss_server_get_stats(ss_server *s, ss_server_stats *out, int reset) {
  if (!s || !out) return ssb::index_error(nullptr, SS_ERR_INVALID_ARGUMENT, "null argument");
  std::lock_guard<std::mutex> lk(s->mu);
  ss_server_stats st{};
  st.submitted = s->n_submitted;
  st.completed = s->n_completed;
  st.failed = s->n_failed;
  st.batches = s->n_batches;
  st.mean_batch = s->n_batches ? (double)s->n_batched / (double)s->n_batches : 0.0;
  st.p50_us = pct(s->latencies, 0.50);
  st.p99_us = pct(s->latencies, 0.99);
  st.p999_us = pct(s->latencies, 0.999);
  st.max_us = s->latencies.empty() ? 0.0 : *std::max_element(s->latencies.begin(),
                                                              s->latencies.end());
  st.slots = (uint32_t)s->slots.size();
  *out = st;
  if (reset) {
    s->n_submitted = s->n_completed = s->n_failed = s->n_batches = s->n_batched = 0;
    s->latencies.clear();
  }
  return SS_OK;
}

void ss_server_destroy(ss_server *s) {
  if (!s) return;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    s->stop = true;
    for (uint64_t t = s->next_dispatch; t < s->next_ticket; ++t) s->req(t).state = kFailed;
    s->next_dispatch = s->next_ticket;
  }
  s->cv_work.notify_all();
  s->cv_done.notify_all();
  if (s->dispatcher.joinable()) s->dispatcher.join();
  int prev = 0;
  cudaGetDevice(&prev);
  cudaSetDevice(s->device);
  s->free_slots();
  cudaSetDevice(prev);
  delete s;
}

}  // extern "C"
