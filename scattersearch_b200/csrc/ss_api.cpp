// Host side of the C ABI declared in include/scattersearch.h.
//
// Owns the device copies of the base rows and the adjacency, plans kernel
// launches, and hands each concurrent caller its own stream and staging
// buffers (the reference shares one ANNSearch between threads that each own
// their visited bitset, tests/search.cpp:75-80; here the per-caller state is
// a SearchCtx borrowed from a pool).
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <mutex>
#include <string>
#include <utility>
#include <vector>

#include "scattersearch.h"
#include "ss_internal.h"

namespace {

thread_local std::string tl_error;
thread_local std::string tl_handle_error_copy;

int fail(std::string *sink, int code, const char *fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  tl_error = buf;
  if (sink) *sink = buf;
  return code;
}

struct DevBuf {
  void *p = nullptr;
  size_t cap = 0;
  DevBuf() = default;
  DevBuf(const DevBuf &) = delete;
  DevBuf &operator=(const DevBuf &) = delete;
  ~DevBuf() {
    if (p) cudaFree(p);
  }
  // Grows to at least `bytes`; new memory is zeroed when `zero` is set.
  cudaError_t ensure(size_t bytes, bool zero = false) {
    if (bytes <= cap) return cudaSuccess;
    if (p) {
      cudaFree(p);
      p = nullptr;
      cap = 0;
    }
    cudaError_t e = cudaMalloc(&p, bytes);
    if (e != cudaSuccess) {
      p = nullptr;
      return e;
    }
    cap = bytes;
    if (zero) e = cudaMemset(p, 0, bytes);
    return e;
  }
  template <class T>
  T *as() const {
    return static_cast<T *>(p);
  }
};

// Per-caller launch state: one stream plus the buffers a search needs.
struct SearchCtx {
  cudaStream_t stream = nullptr;
  DevBuf q, ids, dists, Ks, Ls, off, counter, status, ndc, hops, spill, bf_q, bf_qpack, bf_cand,
      bf_err;
  DevBuf marks, mark_epoch;  // the warp kernel's per-team visited marks (see visited_marks)
  std::vector<int32_t> h_status;
  ~SearchCtx() {
    if (stream) cudaStreamDestroy(stream);
  }
};

uint32_t round_up(uint32_t x, uint32_t m) { return (x + m - 1) / m * m; }

}  // namespace

struct ss_index {
  int device = 0;
  uint32_t dim = 0, n = 0, nb = 0;
  int metric = 0;
  int sm_count = 0;
  DevBuf base;
  DevBuf adj;
  uint32_t rstride = 0, max_deg = 0, ep = 0;
  bool has_graph = false;
  bool row_dups = true;  // some adjacency row repeats an id (found when the graph is set)

  std::mutex mu;  // guards err, contexts
  std::string err;
  std::vector<std::unique_ptr<SearchCtx>> ctx_all;
  std::vector<SearchCtx *> ctx_free;

  std::mutex dev_mu;  // device-batch scratch
  SearchCtx dev_ctx;
  uint32_t dev_last_nq = 0;

  // squared row norms (L2) and the base rows in packed tensor-core tiles for
  // the brute force, built on first use
  std::mutex norm_mu;
  DevBuf xnorm, bpack;
  bool have_norms = false, have_bpack = false;
  // recorded after the kernels that built them; later brute-force calls on
  // any stream wait for it
  cudaEvent_t bf_ready = nullptr;
  ~ss_index() {
    if (bf_ready) cudaEventDestroy(bf_ready);
  }

  // launch tuning (set by the autotuner through ss_set_tuning); 0 = automatic
  int warps_per_block = 0;
  int hash_cap_override = 0;
  int blocks_per_sm_cap = 0;
  int shared_stages = 0;  // row stages shared by a CTA's teams (0 = one per team)
  int stage_rows = 0;     // rows per row stage (0 = 16)
  int row_copy = SS_ROW_COPY_AUTO;  // how row stages are filled (ss_set_row_copy)
  int visited_marks = SS_VISITED_MARKS_AUTO;  // ss_set_visited_marks

  ssb::GraphView view() const {
    ssb::GraphView g;
    g.base = base.as<const float>();
    g.adj = adj.as<const uint32_t>();
    g.n = n;
    g.dim = dim;
    g.nb = nb;
    g.rstride = rstride;
    g.ep = ep;
    g.metric = metric;
    g.row_dups = row_dups ? 1u : 0u;
    return g;
  }
};

namespace {

int cuda_fail(ss_index *h, cudaError_t e, const char *what) {
  return fail(h ? &h->err : nullptr, SS_ERR_CUDA, "%s: %s", what, cudaGetErrorString(e));
}

int set_err(ss_index *h, int code, const char *fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  if (h) {
    std::lock_guard<std::mutex> lk(h->mu);
    return fail(&h->err, code, "%s", buf);
  }
  return fail(nullptr, code, "%s", buf);
}

#define SS_CUDA(h, call, what)                         \
  do {                                                 \
    cudaError_t e_ = (call);                           \
    if (e_ != cudaSuccess) {                           \
      std::lock_guard<std::mutex> lk_((h)->mu);        \
      return cuda_fail((h), e_, what);                 \
    }                                                  \
  } while (0)

struct DeviceGuard {
  int prev = -1;
  explicit DeviceGuard(int dev) {
    cudaGetDevice(&prev);
    if (prev != dev) cudaSetDevice(dev);
  }
  ~DeviceGuard() {
    int cur = -1;
    cudaGetDevice(&cur);
    if (prev >= 0 && cur != prev) cudaSetDevice(prev);
  }
};

SearchCtx *acquire_ctx(ss_index *h) {
  std::lock_guard<std::mutex> lk(h->mu);
  if (!h->ctx_free.empty()) {
    SearchCtx *c = h->ctx_free.back();
    h->ctx_free.pop_back();
    return c;
  }
  auto c = std::make_unique<SearchCtx>();
  if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess) return nullptr;
  SearchCtx *raw = c.get();
  h->ctx_all.push_back(std::move(c));
  return raw;
}

void release_ctx(ss_index *h, SearchCtx *c) {
  std::lock_guard<std::mutex> lk(h->mu);
  h->ctx_free.push_back(c);
}

struct CtxLease {
  ss_index *h;
  SearchCtx *c;
  CtxLease(ss_index *hh) : h(hh), c(acquire_ctx(hh)) {}
  ~CtxLease() {
    if (c) release_ctx(h, c);
  }
};

uint32_t spill_words(const ss_index *h) { return (h->n + 31) / 32; }

int check_search_args(ss_index *h, int K, int L) {
  if (!h) return fail(nullptr, SS_ERR_INVALID_ARGUMENT, "null index handle");
  if (!h->has_graph) return set_err(h, SS_ERR_NO_GRAPH, "no graph loaded");
  if (K < 1 || L < 1 || K > L)
    return set_err(h, SS_ERR_INVALID_ARGUMENT, "need 1 <= K <= L (got K=%d, L=%d)", K, L);
  if (L > SS_MAX_L) return set_err(h, SS_ERR_UNSUPPORTED, "L=%d exceeds SS_MAX_L=%d", L, SS_MAX_L);
  return SS_OK;
}

// Error for a batch from its counts of failed queries per status code
// (counts[c] = queries with status c, 1 <= c < kStatusKinds) and the index
// of the first failed query.  The most severe kind present decides the code.
int status_counts_to_error(ss_index *h, const uint32_t *counts, uint32_t first) {
  const uint32_t bad = counts[ssb::kStatusBadArgs], hop = counts[ssb::kStatusHopLimit];
  const uint32_t full = counts[ssb::kStatusVisitedFull];
  const uint32_t timeout = counts[ssb::kStatusStageTimeout];
  if (timeout)
    return set_err(h, SS_ERR_TIMEOUT,
                   "%u queries gave up waiting for their row copies (first failed query: %u); "
                   "results are invalid", timeout, first);
  if (hop)
    return set_err(h, SS_ERR_SEARCH_LIMIT, "%u queries hit the hop limit (first failed query: %u)",
                   hop, first);
  if (full)
    return set_err(h, SS_ERR_SEARCH_LIMIT,
                   "%u queries overflowed the visited table (first failed query: %u)", full, first);
  if (bad)
    return set_err(h, SS_ERR_INVALID_ARGUMENT, "%u queries had invalid K/L (first failed query: %u)",
                   bad, first);
  return SS_OK;
}

int status_to_error(ss_index *h, const int32_t *st, uint32_t nq) {
  uint32_t counts[ssb::kStatusKinds] = {};
  uint32_t first = 0, failed = 0;
  for (uint32_t i = 0; i < nq; ++i) {
    if (st[i] != ssb::kStatusOk) {
      if (failed++ == 0) first = i;
      // an unknown code counts as invalid arguments
      ++counts[st[i] > 0 && st[i] < ssb::kStatusKinds ? st[i] : ssb::kStatusBadArgs];
    }
  }
  return failed ? status_counts_to_error(h, counts, first) : SS_OK;
}

// Persistent grid size for the warp kernel: every SM filled, never more
// teams than queries.
int persistent_blocks(ss_index *h, const ssb::SmemPlan &p, int wpb, uint32_t nq) {
  int per_sm = ssb::warp_search_occupancy(h->view(), p, wpb);
  if (per_sm <= 0) return 0;
  if (h->blocks_per_sm_cap > 0) per_sm = std::min(per_sm, h->blocks_per_sm_cap);
  long full = (long)per_sm * h->sm_count;
  long need = ((long)nq + wpb - 1) / wpb;
  return (int)std::max(1L, std::min(full, need));
}

// Row stages shared by a CTA of `wpb` teams under the tuning of `h` (0 =
// a private stage per team; sharing needs fewer stages than teams).
int stages_for(const ss_index *h, int wpb) {
  return h->shared_stages > 0 && h->shared_stages < wpb ? h->shared_stages : 0;
}

// Query teams per CTA: the tuned value when set, else the candidate (1, 2,
// 4, 8) that keeps the most teams resident per SM (ties: larger CTAs).  The
// plan's stage layout is set to match.
int choose_wpb(ss_index *h, ssb::SmemPlan &p, bool tuned = true) {
  auto stages = [&](int w) { return tuned ? stages_for(h, w) : 0; };
  auto fits = [&](int w) {
    ssb::SmemPlan q = p;
    ssb::share_stages(q, stages(w));
    return ssb::warp_search_smem_bytes(q, w) <= 227 * 1024;
  };
  if (tuned && h->warps_per_block > 0) {
    int wpb = h->warps_per_block;
    while (wpb > 1 && !fits(wpb)) wpb >>= 1;
    ssb::share_stages(p, stages(wpb));
    return wpb;
  }
  int best = 1, best_teams = -1;
  for (int w = 1; w <= 8; w <<= 1) {
    if (!fits(w)) break;
    const int teams = ssb::warp_search_occupancy(h->view(), p, w) * w;
    if (teams >= best_teams) {
      best_teams = teams;
      best = w;
    }
  }
  ssb::share_stages(p, stages(best));
  return best;
}

int small_hash_cap(int L_max);

// Plans a warp-kernel launch of nq queries.  The latency layout (one 32-row
// stage and a large visited table per team, untuned CTA size) is taken when
// it fits in shared memory and nq is at most `small_limit` -- or, with
// small_limit 0, when every query of the launch can be resident at once in
// it: all queries then run together in either layout, and this one finishes
// each sooner.  Otherwise the tuned (or automatic) layout is used.  Returns
// the plan; *wpb receives the teams per CTA.
ssb::SmemPlan plan_launch(ss_index *h, const ssb::GraphView &g, int L_max, uint32_t nq,
                          uint32_t small_limit, int *wpb) {
  {
    ssb::SmemPlan p = ssb::plan_warp_smem(g, L_max, small_hash_cap(L_max), 32);
    const int w = choose_wpb(h, p, false);
    if (ssb::warp_search_smem_bytes(p, w) <= 227 * 1024) {
      uint32_t limit = small_limit;
      if (limit == 0) {
        const int per_sm = ssb::warp_search_occupancy(g, p, w);
        limit = (uint32_t)std::max(per_sm, 0) * (uint32_t)w * (uint32_t)h->sm_count;
      }
      if (nq <= limit) {
        *wpb = w;
        if (h->row_copy == SS_ROW_COPY_BULK) p.gather = 0;
        return p;
      }
    }
  }
  ssb::SmemPlan p = ssb::plan_warp_smem(g, L_max, h->hash_cap_override, h->stage_rows);
  *wpb = choose_wpb(h, p, true);
  if (h->row_copy == SS_ROW_COPY_BULK) p.gather = 0;
  return p;
}

// Launches whose queries all fit on the GPU at once in the latency layout
// (plan_launch with limit 0) take it whatever the tuning, which is chosen
// for large batches where shared memory per team sets how many queries run
// at once.  Each team then gets a 32-row stage (every fresh row of a hop
// arrives in one copy round trip), a visited table large enough to forget
// almost nothing (fewer repeated evaluations), and the CTA size that keeps
// the most teams resident.  The serving loop runs a few launch slots at
// once, so its launches use a fixed limit: four slots of 128 requests take
// 512 teams, and about 590 fit at L = 400.
constexpr uint32_t kSmallLaunch = 0;
constexpr uint32_t kServerSmallLaunch = 128;
int small_hash_cap(int L_max) {
  uint32_t slots = 1024;
  while (slots < 16384u && slots < (uint32_t)L_max * 20u) slots <<= 1;
  return (int)slots;
}

// Bytes of the warp kernel's visited marks per team slot: one per base row,
// rounded up to 16 (the kernel clears them with 16-byte stores).
uint32_t mark_stride(const ss_index *h) { return round_up(h->n, 16); }

// Whether `bytes` of new visited marks may be allocated: at most a quarter
// of the free device memory and 16 GB.
bool marks_fit(size_t bytes) {
  size_t free_b = 0, total_b = 0;
  if (cudaMemGetInfo(&free_b, &total_b) != cudaSuccess) return false;
  return bytes <= free_b / 4 && bytes <= (16ull << 30);
}

// Points a persistent launch of `slots` team slots at the visited marks of
// context `c`, allocating (or growing) them on first use; leaves a.marks
// null when they are off or do not fit.  Marks and epochs are cleared
// together whenever either is reallocated, so no stale mark can equal a new
// epoch.
int attach_marks(ss_index *h, SearchCtx *c, size_t slots, ssb::BatchArgs &a,
                 cudaStream_t stream) {
  a.marks = nullptr;
  a.mark_epoch = nullptr;
  a.mark_stride = 0;
  if (h->visited_marks != SS_VISITED_MARKS_AUTO || slots == 0) return SS_OK;
  const size_t mb = slots * mark_stride(h), eb = slots * 4;
  if (c->marks.cap < mb || c->mark_epoch.cap < eb) {
    if (!marks_fit(mb > c->marks.cap ? mb - c->marks.cap : 0)) return SS_OK;
    SS_CUDA(h, c->marks.ensure(mb), "visited marks allocation");
    SS_CUDA(h, c->mark_epoch.ensure(eb), "visited marks allocation");
    SS_CUDA(h, cudaMemsetAsync(c->marks.p, 0, c->marks.cap, stream), "visited marks clear");
    SS_CUDA(h, cudaMemsetAsync(c->mark_epoch.p, 0, c->mark_epoch.cap, stream),
            "visited marks clear");
  }
  a.marks = c->marks.as<uint8_t>();
  a.mark_epoch = c->mark_epoch.as<uint32_t>();
  a.mark_stride = mark_stride(h);
  return SS_OK;
}

// Core batched launch into caller-provided device buffers on `stream`.
int launch_batch(ss_index *h, SearchCtx *c, const float *d_q, uint32_t nq, const int32_t *d_K,
                 const int32_t *d_L, const int64_t *d_off, int K0, int L0, int L_max,
                 uint32_t *d_ids, float *d_dists, uint32_t *d_ndc, uint32_t *d_hops,
                 cudaStream_t stream, bool persistent) {
  ssb::GraphView g = h->view();
  int wpb = 1;
  ssb::SmemPlan plan = plan_launch(h, g, L_max, nq, kSmallLaunch, &wpb);
  if (ssb::warp_search_smem_bytes(plan, wpb) > 227 * 1024)
    return set_err(h, SS_ERR_UNSUPPORTED, "L=%d needs %u bytes of shared memory per query",
                   L_max, plan.words_per_team * 4);
  int blocks = persistent ? persistent_blocks(h, plan, wpb, nq)
                          : (int)((nq + (uint32_t)wpb - 1) / (uint32_t)wpb);
  if (blocks <= 0) return set_err(h, SS_ERR_UNSUPPORTED, "search kernel cannot be resident");
  SS_CUDA(h, c->status.ensure((size_t)std::max(nq, 1u) * 4), "status allocation");
  SS_CUDA(h, c->counter.ensure(16), "counter allocation");
  ssb::BatchArgs a{};
  a.queries = d_q;
  a.qstride = h->dim;
  a.nq = nq;
  a.Ks = d_K;
  a.Ls = d_L;
  a.K0 = K0;
  a.L0 = L0;
  a.out_off = d_off;
  a.ids = d_ids;
  a.dists = d_dists;
  a.ndc = d_ndc;
  a.hops = d_hops;
  a.status = c->status.as<int32_t>();
  a.work_counter = persistent ? c->counter.as<uint32_t>() : nullptr;
  a.max_hops = h->n + 1;
  if (persistent) {
    const int rc = attach_marks(h, c, (size_t)blocks * (size_t)wpb, a, stream);
    if (rc) return rc;
  }
  if (persistent) SS_CUDA(h, cudaMemsetAsync(c->counter.p, 0, 4, stream), "counter reset");
  SS_CUDA(h, cudaMemsetAsync(c->status.p, 0, (size_t)nq * 4, stream), "status reset");
  SS_CUDA(h, ssb::launch_warp_search(g, a, plan, wpb, blocks, stream), "search launch");
  return SS_OK;
}

int launch_intra(ss_index *h, SearchCtx *c, const float *d_q, uint32_t nq, int K, int L, int W,
                 uint32_t *d_ids, float *d_dists, uint32_t *d_ndc, uint32_t *d_hops,
                 cudaStream_t stream) {
  ssb::GraphView g = h->view();
  ssb::SmemPlan plan = ssb::plan_intra_smem(g, L, W, h->hash_cap_override);
  if ((size_t)plan.words_per_team * 4 > 227 * 1024)
    return set_err(h, SS_ERR_UNSUPPORTED, "L=%d with %d warps needs %u bytes of shared memory",
                   L, W, plan.words_per_team * 4);
  SS_CUDA(h, c->spill.ensure((size_t)std::max(nq, 1u) * spill_words(h) * 4, true),
          "spill bitset allocation");
  SS_CUDA(h, c->status.ensure((size_t)std::max(nq, 1u) * 4), "status allocation");
  ssb::BatchArgs a{};
  a.queries = d_q;
  a.qstride = h->dim;
  a.nq = nq;
  a.K0 = K;
  a.L0 = L;
  a.ids = d_ids;
  a.dists = d_dists;
  a.ndc = d_ndc;
  a.hops = d_hops;
  a.status = c->status.as<int32_t>();
  a.spill_bits = c->spill.as<uint32_t>();
  a.spill_words = spill_words(h);
  a.max_hops = h->n + 1;
  SS_CUDA(h, cudaMemsetAsync(c->status.p, 0, (size_t)nq * 4, stream), "status reset");
  SS_CUDA(h, ssb::launch_intra_search(g, a, plan, W, stream), "intra search launch");
  return SS_OK;
}

int launch_scatter(ss_index *h, SearchCtx *c, const float *d_q, uint32_t nq, int K, int L, int W,
                   int et, uint64_t seed, uint32_t *d_ids, float *d_dists, uint32_t *d_ndc,
                   uint32_t *d_hops, cudaStream_t stream, uint32_t *d_ndc_max = nullptr,
                   uint32_t *d_ndc_min = nullptr) {
  ssb::GraphView g = h->view();
  ssb::SmemPlan plan = ssb::plan_scatter_smem(g, L, W);
  if (ssb::scatter_smem_bytes(plan, W) > 227 * 1024)
    return set_err(h, SS_ERR_UNSUPPORTED, "L=%d with %d warps needs %zu bytes of shared memory",
                   L, W, ssb::scatter_smem_bytes(plan, W));
  SS_CUDA(h, c->spill.ensure((size_t)std::max(nq, 1u) * spill_words(h) * 4, true),
          "spill bitset allocation");
  SS_CUDA(h, c->status.ensure((size_t)std::max(nq, 1u) * 4), "status allocation");
  ssb::BatchArgs a{};
  a.queries = d_q;
  a.qstride = h->dim;
  a.nq = nq;
  a.K0 = K;
  a.L0 = L;
  a.ids = d_ids;
  a.dists = d_dists;
  a.ndc = d_ndc;
  a.hops = d_hops;
  a.ndc_max = d_ndc_max;
  a.ndc_min = d_ndc_min;
  a.status = c->status.as<int32_t>();
  a.spill_bits = c->spill.as<uint32_t>();
  a.spill_words = spill_words(h);
  a.max_hops = h->n + 1;
  SS_CUDA(h, cudaMemsetAsync(c->status.p, 0, (size_t)nq * 4, stream), "status reset");
  SS_CUDA(h, ssb::launch_scatter_search(g, a, plan, W, et, seed, stream), "scatter launch");
  return SS_OK;
}

int check_scatter_args(ss_index *h, int K, int L, int W) {
  int rc = check_search_args(h, K, L);
  if (rc) return rc;
  if (W < 1 || W > SS_SCATTER_MAX_WARPS)
    return set_err(h, SS_ERR_INVALID_ARGUMENT, "num_threads=%d outside 1..%d", W,
                   SS_SCATTER_MAX_WARPS);
  if (L > 512) return set_err(h, SS_ERR_UNSUPPORTED, "the scatter search takes L <= 512");
  return SS_OK;
}

int upload_graph(ss_index *h, const std::vector<uint32_t> &adj, uint32_t rstride, uint32_t ep,
                 uint32_t max_deg) {
  DeviceGuard dg(h->device);
  SS_CUDA(h, h->adj.ensure(adj.size() * 4), "adjacency allocation");
  SS_CUDA(h, cudaMemcpy(h->adj.p, adj.data(), adj.size() * 4, cudaMemcpyHostToDevice),
          "adjacency upload");
  // rows that repeat an id need the kernels' in-row duplicate checks
  DevBuf flag;
  SS_CUDA(h, flag.ensure(4, true), "row check allocation");
  SS_CUDA(h, ssb::launch_row_repeats(h->adj.as<uint32_t>(), h->n, rstride, flag.as<uint32_t>(), 0),
          "row check");
  uint32_t dups = 1;
  SS_CUDA(h, cudaMemcpy(&dups, flag.p, 4, cudaMemcpyDeviceToHost), "row check");
  h->rstride = rstride;
  h->ep = ep;
  h->max_deg = max_deg;
  h->row_dups = dups != 0;
  h->has_graph = true;
  return SS_OK;
}

int create_common(uint32_t dim, uint32_t num, const float *src, bool src_on_device, int metric,
                  int device, ss_index **out) {
  if (!out) return fail(nullptr, SS_ERR_INVALID_ARGUMENT, "null output handle");
  *out = nullptr;
  if (dim == 0 || num == 0 || !src)
    return fail(nullptr, SS_ERR_INVALID_ARGUMENT, "dim, num and base must be nonzero");
  if (num >= 0x80000000u) return fail(nullptr, SS_ERR_UNSUPPORTED, "num must be < 2^31");
  if (metric != SS_METRIC_L2 && metric != SS_METRIC_INNER_PRODUCT)
    return fail(nullptr, SS_ERR_INVALID_ARGUMENT, "unknown metric %d", metric);
  int dev = device;
  if (dev < 0 && cudaGetDevice(&dev) != cudaSuccess) dev = 0;
  int ndev = 0;
  cudaError_t e = cudaGetDeviceCount(&ndev);
  if (e != cudaSuccess || ndev == 0)
    return fail(nullptr, SS_ERR_CUDA, "no CUDA device: %s", cudaGetErrorString(e));
  if (dev >= ndev) return fail(nullptr, SS_ERR_INVALID_ARGUMENT, "device %d out of range", dev);
  auto h = std::make_unique<ss_index>();
  h->device = dev;
  h->dim = dim;
  h->n = num;
  h->nb = (dim + 7) / 8;
  h->metric = metric;
  DeviceGuard dg(dev);
  cudaDeviceGetAttribute(&h->sm_count, cudaDevAttrMultiProcessorCount, dev);
  const size_t pitch = (size_t)h->nb * 8 * 4;
  e = h->base.ensure(pitch * num);
  if (e != cudaSuccess)
    return fail(nullptr, SS_ERR_OUT_OF_MEMORY, "base allocation (%zu bytes): %s", pitch * num,
                cudaGetErrorString(e));
  if (pitch != (size_t)dim * 4) {
    e = cudaMemset(h->base.p, 0, pitch * num);
    if (e != cudaSuccess) return fail(nullptr, SS_ERR_CUDA, "base clear: %s", cudaGetErrorString(e));
  }
  e = cudaMemcpy2D(h->base.p, pitch, src, (size_t)dim * 4, (size_t)dim * 4, num,
                   src_on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice);
  if (e != cudaSuccess) return fail(nullptr, SS_ERR_CUDA, "base upload: %s", cudaGetErrorString(e));
  e = cudaDeviceSynchronize();
  if (e != cudaSuccess) return fail(nullptr, SS_ERR_CUDA, "base upload: %s", cudaGetErrorString(e));
  *out = h.release();
  return SS_OK;
}

}  // namespace

// Host-side hooks for the serving loop (ss_server.cpp), declared in
// ss_internal.h.
namespace ssb {

int index_device(const ss_index *h) { return h->device; }
uint32_t index_dim(const ss_index *h) { return h->dim; }
bool index_ready(const ss_index *h) { return h && h->has_graph; }

int index_error(ss_index *h, int code, const char *msg) { return set_err(h, code, "%s", msg); }

int server_launch(ss_index *h, const float *d_q, uint32_t nq, const int32_t *d_K,
                  const int32_t *d_L, const int64_t *d_off, int L_max, uint32_t *d_ids,
                  float *d_dists, int32_t *d_status, uint32_t *d_counter, cudaStream_t stream) {
  ssb::GraphView g = h->view();
  int wpb = 1;
  ssb::SmemPlan plan = plan_launch(h, g, L_max, nq, kServerSmallLaunch, &wpb);
  if (ssb::warp_search_smem_bytes(plan, wpb) > 227 * 1024)
    return set_err(h, SS_ERR_UNSUPPORTED, "L=%d needs %u bytes of shared memory per query",
                   L_max, plan.words_per_team * 4);
  const int blocks = persistent_blocks(h, plan, wpb, nq);
  if (blocks <= 0) return set_err(h, SS_ERR_UNSUPPORTED, "search kernel cannot be resident");
  ssb::BatchArgs a{};
  a.queries = d_q;
  a.qstride = h->dim;
  a.nq = nq;
  a.Ks = d_K;
  a.Ls = d_L;
  a.out_off = d_off;
  a.ids = d_ids;
  a.dists = d_dists;
  a.status = d_status;
  a.work_counter = d_counter;
  a.max_hops = h->n + 1;
  SS_CUDA(h, cudaMemsetAsync(d_counter, 0, 4, stream), "counter reset");
  SS_CUDA(h, cudaMemsetAsync(d_status, 0, (size_t)nq * 4, stream), "status reset");
  SS_CUDA(h, ssb::launch_warp_search(g, a, plan, wpb, blocks, stream), "search launch");
  return SS_OK;
}

}  // namespace ssb

extern "C" {

const char *ss_version(void) { return "scattersearch_b200 0.1 sm_100a"; }

const char *ss_last_error(const ss_index *h) {
  if (!h) return tl_error.c_str();
  auto *hh = const_cast<ss_index *>(h);
  std::lock_guard<std::mutex> lk(hh->mu);
  tl_handle_error_copy = hh->err;
  return tl_handle_error_copy.c_str();
}

void ss_free(void *p) { free(p); }

int ss_create(uint32_t dim, uint32_t num, const float *base_host, int metric, int device,
              ss_index **out) {
  return create_common(dim, num, base_host, false, metric, device, out);
}

int ss_create_from_device(uint32_t dim, uint32_t num, const float *base_dev, int metric,
                          int device, ss_index **out) {
  return create_common(dim, num, base_dev, true, metric, device, out);
}

void ss_destroy(ss_index *h) {
  if (!h) return;
  DeviceGuard dg(h->device);
  cudaDeviceSynchronize();
  delete h;
}

int ss_set_graph(ss_index *h, const uint32_t *adj, uint32_t n, uint32_t rstride,
                 uint32_t entry_point) {
  if (!h) return fail(nullptr, SS_ERR_INVALID_ARGUMENT, "null index handle");
  if (!adj || rstride == 0) return set_err(h, SS_ERR_INVALID_ARGUMENT, "empty adjacency");
  if (n != h->n) return set_err(h, SS_ERR_FORMAT, "graph has %u nodes, index has %u", n, h->n);
  if (entry_point >= n)
    return set_err(h, SS_ERR_FORMAT, "entry point %u out of range (n=%u)", entry_point, n);
  uint32_t max_deg = 0;
  for (uint32_t i = 0; i < n; ++i) {
    const uint32_t *row = adj + (size_t)i * rstride;
    uint32_t d = 0;
    while (d < rstride && row[d] != ssb::kNoneId) {
      if (row[d] >= n)
        return set_err(h, SS_ERR_FORMAT, "node %u has neighbour id %u >= n", i, row[d]);
      ++d;
    }
    for (uint32_t m = d; m < rstride; ++m)
      if (row[m] != ssb::kNoneId)
        return set_err(h, SS_ERR_FORMAT, "node %u: padding must only follow the neighbours", i);
    max_deg = std::max(max_deg, d);
  }
  if (max_deg > SS_MAX_DEGREE)
    return set_err(h, SS_ERR_UNSUPPORTED, "degree %u exceeds SS_MAX_DEGREE=%d", max_deg,
                   SS_MAX_DEGREE);
  const uint32_t rs = std::max(8u, round_up(max_deg, 8));
  std::vector<uint32_t> packed((size_t)n * rs, ssb::kNoneId);
  for (uint32_t i = 0; i < n; ++i)
    memcpy(&packed[(size_t)i * rs], adj + (size_t)i * rstride, std::min(rs, rstride) * 4);
  return upload_graph(h, packed, rs, entry_point, max_deg);
}

int ss_load_graph(ss_index *h, const char *path) {
  if (!h) return fail(nullptr, SS_ERR_INVALID_ARGUMENT, "null index handle");
  if (!path) return set_err(h, SS_ERR_INVALID_ARGUMENT, "null path");
  FILE *f = fopen(path, "rb");
  if (!f) return set_err(h, SS_ERR_IO, "cannot open graph file %s", path);
  uint32_t hdr[2];
  if (fread(hdr, 4, 2, f) != 2) {
    fclose(f);
    return set_err(h, SS_ERR_FORMAT, "%s: missing NSG header", path);
  }
  const uint32_t ep = hdr[1];
  std::vector<std::vector<uint32_t>> rows;
  rows.reserve(h->n);
  uint32_t max_deg = 0;
  for (;;) {
    uint32_t k;
    const size_t got = fread(&k, 4, 1, f);
    if (got != 1) break;  // end of file between records
    if (k > SS_MAX_DEGREE) {
      fclose(f);
      return set_err(h, SS_ERR_UNSUPPORTED, "%s: node %zu has degree %u > SS_MAX_DEGREE", path,
                     rows.size(), k);
    }
    std::vector<uint32_t> r(k);
    if (k && fread(r.data(), 4, k, f) != k) {
      fclose(f);
      return set_err(h, SS_ERR_FORMAT, "%s: truncated record for node %zu", path, rows.size());
    }
    max_deg = std::max(max_deg, k);
    rows.push_back(std::move(r));
    if (rows.size() > h->n) break;
  }
  fclose(f);
  if (rows.size() != h->n)
    return set_err(h, SS_ERR_FORMAT, "%s: %zu node records, index has %u", path, rows.size(), h->n);
  if (ep >= h->n) return set_err(h, SS_ERR_FORMAT, "%s: entry point %u out of range", path, ep);
  const uint32_t rs = std::max(8u, round_up(max_deg, 8));
  std::vector<uint32_t> packed((size_t)h->n * rs, ssb::kNoneId);
  for (uint32_t i = 0; i < h->n; ++i) {
    for (size_t m = 0; m < rows[i].size(); ++m) {
      if (rows[i][m] >= h->n)
        return set_err(h, SS_ERR_FORMAT, "%s: node %u has neighbour id %u >= n", path, i,
                       rows[i][m]);
      packed[(size_t)i * rs + m] = rows[i][m];
    }
  }
  return upload_graph(h, packed, rs, ep, max_deg);
}

int ss_graph_info(const ss_index *h, uint32_t *n, uint32_t *max_degree, uint32_t *entry_point,
                  uint32_t *rstride) {
  if (!h) return fail(nullptr, SS_ERR_INVALID_ARGUMENT, "null index handle");
  if (n) *n = h->n;
  if (max_degree) *max_degree = h->max_deg;
  if (entry_point) *entry_point = h->ep;
  if (rstride) *rstride = h->rstride;
  return h->has_graph ? SS_OK : SS_ERR_NO_GRAPH;
}

int ss_get_graph(ss_index *h, uint32_t *adj, uint32_t rstride) {
  if (!h) return fail(nullptr, SS_ERR_INVALID_ARGUMENT, "null index handle");
  if (!h->has_graph) return set_err(h, SS_ERR_NO_GRAPH, "no graph loaded");
  if (!adj || rstride < h->max_deg)
    return set_err(h, SS_ERR_INVALID_ARGUMENT, "rstride %u below max degree %u", rstride,
                   h->max_deg);
  DeviceGuard dg(h->device);
  std::vector<uint32_t> tmp((size_t)h->n * h->rstride);
  SS_CUDA(h, cudaMemcpy(tmp.data(), h->adj.p, tmp.size() * 4, cudaMemcpyDeviceToHost),
          "adjacency download");
  for (uint32_t i = 0; i < h->n; ++i)
    for (uint32_t m = 0; m < rstride; ++m)
      adj[(size_t)i * rstride + m] = m < h->rstride ? tmp[(size_t)i * h->rstride + m] : ssb::kNoneId;
  return SS_OK;
}

int ss_search(ss_index *h, const float *query, int K, int L, uint32_t *ids, float *dists) {
  int rc = check_search_args(h, K, L);
  if (rc) return rc;
  if (!query || !ids) return set_err(h, SS_ERR_INVALID_ARGUMENT, "null query or ids");
  DeviceGuard dg(h->device);
  CtxLease lease(h);
  SearchCtx *c = lease.c;
  if (!c) return set_err(h, SS_ERR_CUDA, "cannot create a stream");
  SS_CUDA(h, c->q.ensure((size_t)h->dim * 4), "query buffer");
  SS_CUDA(h, c->ids.ensure((size_t)K * 4), "ids buffer");
  SS_CUDA(h, c->dists.ensure((size_t)K * 4), "dists buffer");
  SS_CUDA(h, cudaMemcpyAsync(c->q.p, query, (size_t)h->dim * 4, cudaMemcpyHostToDevice, c->stream),
          "query upload");
  rc = launch_batch(h, c, c->q.as<float>(), 1, nullptr, nullptr, nullptr, K, L, L,
                    c->ids.as<uint32_t>(), c->dists.as<float>(), nullptr, nullptr, c->stream, false);
  if (rc) return rc;
  int32_t st = 0;
  SS_CUDA(h, cudaMemcpyAsync(ids, c->ids.p, (size_t)K * 4, cudaMemcpyDeviceToHost, c->stream),
          "ids download");
  if (dists)
    SS_CUDA(h, cudaMemcpyAsync(dists, c->dists.p, (size_t)K * 4, cudaMemcpyDeviceToHost, c->stream),
            "dists download");
  SS_CUDA(h, cudaMemcpyAsync(&st, c->status.p, 4, cudaMemcpyDeviceToHost, c->stream),
          "status download");
  SS_CUDA(h, cudaStreamSynchronize(c->stream), "search");
  return status_to_error(h, &st, 1);
}

static int batch_common(ss_index *h, const float *queries, uint32_t nq, const int32_t *Ks,
                        const int32_t *Ls, int K, int L, uint32_t *ids, float *dists) {
  if (!h) return fail(nullptr, SS_ERR_INVALID_ARGUMENT, "null index handle");
  if (!h->has_graph) return set_err(h, SS_ERR_NO_GRAPH, "no graph loaded");
  if (nq == 0) return SS_OK;
  if (!queries || !ids) return set_err(h, SS_ERR_INVALID_ARGUMENT, "null queries or ids");
  int L_max = L;
  size_t total = (size_t)nq * (size_t)K;
  std::vector<int64_t> off;
  if (Ks) {
    L_max = 0;
    total = 0;
    off.resize(nq);
    for (uint32_t i = 0; i < nq; ++i) {
      int rc = check_search_args(h, Ks[i], Ls[i]);
      if (rc) return rc;
      off[i] = (int64_t)total;
      total += (size_t)Ks[i];
      L_max = std::max(L_max, (int)Ls[i]);
    }
  } else {
    int rc = check_search_args(h, K, L);
    if (rc) return rc;
  }
  DeviceGuard dg(h->device);
  CtxLease lease(h);
  SearchCtx *c = lease.c;
  if (!c) return set_err(h, SS_ERR_CUDA, "cannot create a stream");
  SS_CUDA(h, c->q.ensure((size_t)nq * h->dim * 4), "query buffer");
  SS_CUDA(h, c->ids.ensure(total * 4), "ids buffer");
  SS_CUDA(h, c->dists.ensure(total * 4), "dists buffer");
  SS_CUDA(h, cudaMemcpyAsync(c->q.p, queries, (size_t)nq * h->dim * 4, cudaMemcpyHostToDevice,
                             c->stream),
          "query upload");
  if (Ks) {
    SS_CUDA(h, c->Ks.ensure((size_t)nq * 4), "K buffer");
    SS_CUDA(h, c->Ls.ensure((size_t)nq * 4), "L buffer");
    SS_CUDA(h, c->off.ensure((size_t)nq * 8), "offset buffer");
    SS_CUDA(h, cudaMemcpyAsync(c->Ks.p, Ks, (size_t)nq * 4, cudaMemcpyHostToDevice, c->stream), "K upload");
    SS_CUDA(h, cudaMemcpyAsync(c->Ls.p, Ls, (size_t)nq * 4, cudaMemcpyHostToDevice, c->stream), "L upload");
    SS_CUDA(h, cudaMemcpyAsync(c->off.p, off.data(), (size_t)nq * 8, cudaMemcpyHostToDevice, c->stream),
            "offset upload");
  }
  int rc = launch_batch(h, c, c->q.as<float>(), nq, Ks ? c->Ks.as<int32_t>() : nullptr,
                        Ks ? c->Ls.as<int32_t>() : nullptr, Ks ? c->off.as<int64_t>() : nullptr,
                        K, L, L_max, c->ids.as<uint32_t>(), c->dists.as<float>(), nullptr, nullptr,
                        c->stream, true);
  if (rc) return rc;
  c->h_status.resize(nq);
  SS_CUDA(h, cudaMemcpyAsync(ids, c->ids.p, total * 4, cudaMemcpyDeviceToHost, c->stream),
          "ids download");
  if (dists)
    SS_CUDA(h, cudaMemcpyAsync(dists, c->dists.p, total * 4, cudaMemcpyDeviceToHost, c->stream),
            "dists download");
  SS_CUDA(h, cudaMemcpyAsync(c->h_status.data(), c->status.p, (size_t)nq * 4,
                             cudaMemcpyDeviceToHost, c->stream),
          "status download");
  SS_CUDA(h, cudaStreamSynchronize(c->stream), "batched search");
  return status_to_error(h, c->h_status.data(), nq);
}

int ss_search_batch(ss_index *h, const float *queries, uint32_t nq, int K, int L, uint32_t *ids,
                    float *dists) {
  return batch_common(h, queries, nq, nullptr, nullptr, K, L, ids, dists);
}

int ss_search_batch_uneven(ss_index *h, const float *queries, uint32_t nq, const int32_t *Ks,
                           const int32_t *Ls, uint32_t *ids, float *dists) {
  if (!Ks || !Ls) return set_err(h, SS_ERR_INVALID_ARGUMENT, "null Ks or Ls");
  return batch_common(h, queries, nq, Ks, Ls, 0, 0, ids, dists);
}

int ss_search_batch_device(ss_index *h, const float *queries, uint32_t nq, const int32_t *Ks,
                           const int32_t *Ls, const int64_t *out_off, int K, int L, int L_max,
                           uint32_t *ids, float *dists, uint32_t *ndc, uint32_t *hops,
                           void *stream) {
  if (!h) return fail(nullptr, SS_ERR_INVALID_ARGUMENT, "null index handle");
  if (!h->has_graph) return set_err(h, SS_ERR_NO_GRAPH, "no graph loaded");
  if (!queries || !ids) return set_err(h, SS_ERR_INVALID_ARGUMENT, "null queries or ids");
  const bool uneven = Ks != nullptr;
  if (uneven != (Ls != nullptr) || uneven != (out_off != nullptr))
    return set_err(h, SS_ERR_INVALID_ARGUMENT, "Ks, Ls and out_off must be given together");
  if (uneven) {
    if (L_max < 1 || L_max > SS_MAX_L)
      return set_err(h, SS_ERR_INVALID_ARGUMENT, "L_max=%d out of range", L_max);
  } else {
    int rc = check_search_args(h, K, L);
    if (rc) return rc;
    L_max = L;
  }
  DeviceGuard dg(h->device);
  std::lock_guard<std::mutex> lk(h->dev_mu);
  h->dev_last_nq = nq;
  if (nq == 0) return SS_OK;
  return launch_batch(h, &h->dev_ctx, queries, nq, Ks, Ls, out_off, K, L, L_max, ids, dists, ndc,
                      hops, static_cast<cudaStream_t>(stream), true);
}

}  // extern "C"

struct ss_plan {
  ss_index *h = nullptr;
  uint32_t nq = 0;
  int32_t *status = nullptr;
  uint32_t *counter = nullptr;
  SearchCtx marks;  // the plan's own visited marks (only marks/mark_epoch are used)
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
};

namespace {
void plan_free(ss_plan *p) {
  if (!p) return;
  if (p->exec) cudaGraphExecDestroy(p->exec);
  if (p->graph) cudaGraphDestroy(p->graph);
  if (p->status) cudaFree(p->status);
  if (p->counter) cudaFree(p->counter);
  delete p;
}
}  // namespace

extern "C" {

int ss_plan_create(ss_index *h, const float *queries, uint32_t nq, int K, int L, uint32_t *ids,
                   float *dists, ss_plan **out) {
  return ss_plan_create_uneven(h, queries, nq, nullptr, nullptr, nullptr, K, L, L, ids, dists, out);
}

int ss_plan_create_uneven(ss_index *h, const float *queries, uint32_t nq, const int32_t *Ks,
                          const int32_t *Ls, const int64_t *out_off, int K, int L, int L_max,
                          uint32_t *ids, float *dists, ss_plan **out) {
  if (!out) return fail(nullptr, SS_ERR_INVALID_ARGUMENT, "null output plan");
  *out = nullptr;
  const bool uneven = Ks != nullptr;
  if (uneven != (Ls != nullptr) || uneven != (out_off != nullptr))
    return set_err(h, SS_ERR_INVALID_ARGUMENT, "Ks, Ls and out_off must be given together");
  int rc = uneven ? check_search_args(h, 1, L_max) : check_search_args(h, K, L);
  if (rc) return rc;
  if (!uneven) L_max = L;
  if (nq == 0 || !queries || !ids)
    return set_err(h, SS_ERR_INVALID_ARGUMENT, "a plan needs nq > 0, queries and ids");
  DeviceGuard dg(h->device);
  auto *p = new ss_plan();
  p->h = h;
  p->nq = nq;
  cudaStream_t cs = nullptr;
  cudaError_t e = cudaMalloc(&p->status, (size_t)nq * 4);
  if (e == cudaSuccess) e = cudaMalloc(&p->counter, 16);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking);
  if (e != cudaSuccess) {
    plan_free(p);
    if (cs) cudaStreamDestroy(cs);
    std::lock_guard<std::mutex> lk(h->mu);
    return cuda_fail(h, e, "plan allocation");
  }
  // Plan the launch outside the capture (occupancy queries and kernel
  // attributes are not stream work).
  ssb::GraphView g = h->view();
  int wpb = 1;
  ssb::SmemPlan plan = plan_launch(h, g, L_max, nq, kSmallLaunch, &wpb);
  const int blocks = persistent_blocks(h, plan, wpb, nq);
  if (ssb::warp_search_smem_bytes(plan, wpb) > 227 * 1024 || blocks <= 0) {
    plan_free(p);
    cudaStreamDestroy(cs);
    return set_err(h, SS_ERR_UNSUPPORTED, "L=%d cannot be planned on this device", L_max);
  }
  ssb::BatchArgs a{};
  a.queries = queries;
  a.qstride = h->dim;
  a.nq = nq;
  a.Ks = Ks;
  a.Ls = Ls;
  a.out_off = out_off;
  a.K0 = K;
  a.L0 = L;
  a.ids = ids;
  a.dists = dists;
  a.status = p->status;
  a.work_counter = p->counter;
  a.max_hops = h->n + 1;
  // marks are allocated and cleared before the capture; the graph only
  // reads and advances them
  rc = attach_marks(h, &p->marks, (size_t)blocks * (size_t)wpb, a, cs);
  if (rc == SS_OK) e = cudaStreamSynchronize(cs);
  if (rc != SS_OK || e != cudaSuccess) {
    plan_free(p);
    cudaStreamDestroy(cs);
    if (rc != SS_OK) return rc;
    std::lock_guard<std::mutex> lk(h->mu);
    return cuda_fail(h, e, "plan visited marks");
  }
  e = cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal);
  if (e == cudaSuccess) {
    cudaError_t e1 = cudaMemsetAsync(p->counter, 0, 4, cs);
    cudaError_t e2 = cudaMemsetAsync(p->status, 0, (size_t)nq * 4, cs);
    cudaError_t e3 = ssb::launch_warp_search(g, a, plan, wpb, blocks, cs);
    e = cudaStreamEndCapture(cs, &p->graph);
    if (e == cudaSuccess) e = e1 != cudaSuccess ? e1 : e2 != cudaSuccess ? e2 : e3;
  }
  if (e == cudaSuccess) e = cudaGraphInstantiate(&p->exec, p->graph, 0);
  cudaStreamDestroy(cs);
  if (e != cudaSuccess) {
    plan_free(p);
    std::lock_guard<std::mutex> lk(h->mu);
    return cuda_fail(h, e, "graph capture of the search launch");
  }
  *out = p;
  return SS_OK;
}

int ss_plan_launch(ss_plan *p, void *stream) {
  if (!p) return fail(nullptr, SS_ERR_INVALID_ARGUMENT, "null plan");
  DeviceGuard dg(p->h->device);
  SS_CUDA(p->h, cudaGraphLaunch(p->exec, static_cast<cudaStream_t>(stream)), "graph launch");
  return SS_OK;
}

int ss_plan_status(ss_plan *p, uint32_t *failed_queries) {
  if (!p || !failed_queries) return fail(nullptr, SS_ERR_INVALID_ARGUMENT, "null argument");
  DeviceGuard dg(p->h->device);
  std::vector<int32_t> st(p->nq);
  SS_CUDA(p->h, cudaMemcpy(st.data(), p->status, (size_t)p->nq * 4, cudaMemcpyDeviceToHost),
          "status download");
  uint32_t bad = 0;
  for (int32_t v : st) bad += v != 0;
  *failed_queries = bad;
  return SS_OK;
}

void ss_plan_destroy(ss_plan *p) {
  if (!p) return;
  DeviceGuard dg(p->h->device);
  cudaDeviceSynchronize();
  plan_free(p);
}

}  // extern "C"

namespace {
// Brute force of nq device queries (row stride `qstride` floats) into device
// ids/dists on `stream`, with scratch from `c`.
int bruteforce_common(ss_index *h, SearchCtx *c, const float *d_queries, size_t qstride,
                      uint32_t nq, int k, uint32_t *d_ids, float *d_dists, cudaStream_t stream) {
  const uint32_t pitch = h->nb * 8;
  const float *xnorm = nullptr;
  const float *bpack = nullptr;
  {
    // the norms and the packed base are built once, on the first caller's
    // stream; every later caller's stream waits for that work
    std::lock_guard<std::mutex> lk(h->norm_mu);
    bool built = false;
    if (h->metric == SS_METRIC_L2 && !h->have_norms) {
      SS_CUDA(h, h->xnorm.ensure((size_t)h->n * 4), "norm buffer");
      SS_CUDA(h, ssb::launch_norms(h->base.as<float>(), h->n, pitch, h->xnorm.as<float>(), stream),
              "norm launch");
      h->have_norms = true;
      built = true;
    }
    if (!h->have_bpack) {
      SS_CUDA(h, h->bpack.ensure(ssb::bruteforce_pack_bytes(h->n, h->dim, true)), "packed base");
      SS_CUDA(h, ssb::launch_pack(h->base.as<float>(), h->n, pitch, h->dim, true,
                                  h->bpack.as<float>(), stream),
              "base packing");
      h->have_bpack = true;
      built = true;
    }
    if (!h->bf_ready)
      SS_CUDA(h, cudaEventCreateWithFlags(&h->bf_ready, cudaEventDisableTiming), "event");
    if (built) SS_CUDA(h, cudaEventRecord(h->bf_ready, stream), "event record");
    else SS_CUDA(h, cudaStreamWaitEvent(stream, h->bf_ready, 0), "event wait");
    if (h->metric == SS_METRIC_L2) xnorm = h->xnorm.as<float>();
    bpack = h->bpack.as<float>();
  }
  ssb::BrutePlan bp = ssb::plan_bruteforce(h->n, nq, k, h->sm_count);
  const uint32_t lists = bp.lists;
  SS_CUDA(h, c->bf_q.ensure((size_t)nq * pitch * 4), "query buffer");
  SS_CUDA(h, c->bf_qpack.ensure(ssb::bruteforce_pack_bytes(nq, h->dim, false)), "packed queries");
  SS_CUDA(h, c->bf_cand.ensure((size_t)nq * lists * bp.list_cap * 8), "candidate buffer");
  SS_CUDA(h, c->bf_err.ensure(4), "error word");
  SS_CUDA(h, cudaMemsetAsync(c->bf_err.p, 0, 4, stream), "error word clear");
  SS_CUDA(h, cudaMemsetAsync(c->bf_q.p, 0, (size_t)nq * pitch * 4, stream), "query clear");
  SS_CUDA(h, cudaMemcpy2DAsync(c->bf_q.p, (size_t)pitch * 4, d_queries, qstride * 4,
                               (size_t)h->dim * 4, nq, cudaMemcpyDeviceToDevice, stream),
          "query copy");
  SS_CUDA(h, ssb::launch_pack(d_queries, nq, (uint32_t)qstride, h->dim, false,
                              c->bf_qpack.as<float>(), stream),
          "query packing");
  ssb::BruteArgs a{};
  a.base = h->base.as<float>();
  a.n = h->n;
  a.nb = h->nb;
  a.queries = c->bf_q.as<float>();
  a.nq = nq;
  a.qpack = c->bf_qpack.as<float>();
  a.bpack = bpack;
  a.kblocks = ssb::bruteforce_kblocks(h->dim);
  a.xnorm = xnorm;
  a.metric = h->metric;
  a.k = k;
  a.C = bp.C;
  a.splits = bp.splits;
  a.rows_per_split = bp.rows_per_split;
  a.lists = lists;
  a.list_stride = bp.list_cap;
  a.cand = c->bf_cand.as<uint64_t>();
  a.ids = d_ids;
  a.dists = d_dists;
  a.err = c->bf_err.as<uint32_t>();
  SS_CUDA(h, ssb::launch_bruteforce(a, h->view(), stream), "brute-force launch");
  return SS_OK;
}

int check_bruteforce_args(ss_index *h, int k) {
  if (!h) return fail(nullptr, SS_ERR_INVALID_ARGUMENT, "null index handle");
  if (k < 1) return set_err(h, SS_ERR_INVALID_ARGUMENT, "need k >= 1 (got %d)", k);
  if (k > ssb::kBruteMaxK)
    return set_err(h, SS_ERR_UNSUPPORTED, "k=%d exceeds the brute force's limit of %d", k,
                   ssb::kBruteMaxK);
  return SS_OK;
}
}  // namespace

extern "C" {

int ss_bruteforce(ss_index *h, const float *queries, uint32_t nq, int k, uint32_t *ids,
                  float *dists) {
  int rc = check_bruteforce_args(h, k);
  if (rc) return rc;
  if (nq == 0) return SS_OK;
  if (!queries || !ids) return set_err(h, SS_ERR_INVALID_ARGUMENT, "null queries or ids");
  DeviceGuard dg(h->device);
  CtxLease lease(h);
  SearchCtx *c = lease.c;
  if (!c) return set_err(h, SS_ERR_CUDA, "cannot create a stream");
  const size_t total = (size_t)nq * k;
  SS_CUDA(h, c->q.ensure((size_t)nq * h->dim * 4), "query buffer");
  SS_CUDA(h, c->ids.ensure(total * 4), "ids buffer");
  SS_CUDA(h, c->dists.ensure(total * 4), "dists buffer");
  SS_CUDA(h, cudaMemcpyAsync(c->q.p, queries, (size_t)nq * h->dim * 4, cudaMemcpyHostToDevice,
                             c->stream),
          "query upload");
  rc = bruteforce_common(h, c, c->q.as<float>(), h->dim, nq, k, c->ids.as<uint32_t>(),
                         c->dists.as<float>(), c->stream);
  if (rc) return rc;
  uint32_t err = 0;
  SS_CUDA(h, cudaMemcpyAsync(ids, c->ids.p, total * 4, cudaMemcpyDeviceToHost, c->stream),
          "ids download");
  if (dists)
    SS_CUDA(h, cudaMemcpyAsync(dists, c->dists.p, total * 4, cudaMemcpyDeviceToHost, c->stream),
            "dists download");
  SS_CUDA(h, cudaMemcpyAsync(&err, c->bf_err.p, 4, cudaMemcpyDeviceToHost, c->stream),
          "error word download");
  SS_CUDA(h, cudaStreamSynchronize(c->stream), "brute force");
  if (err)
    return set_err(h, SS_ERR_TIMEOUT, "a brute-force pipeline wait ran out; results are invalid");
  return SS_OK;
}

int ss_bruteforce_device(ss_index *h, const float *queries, uint32_t nq, int k, uint32_t *ids,
                         float *dists, void *stream) {
  int rc = check_bruteforce_args(h, k);
  if (rc) return rc;
  if (nq == 0) return SS_OK;
  if (!queries || !ids) return set_err(h, SS_ERR_INVALID_ARGUMENT, "null queries or ids");
  DeviceGuard dg(h->device);
  std::lock_guard<std::mutex> lk(h->dev_mu);
  return bruteforce_common(h, &h->dev_ctx, queries, h->dim, nq, k, ids, dists,
                           static_cast<cudaStream_t>(stream));
}

int ss_search_scatter_batch(ss_index *h, const float *queries, uint32_t nq, int K, int L,
                            int num_threads, int early_termination, uint64_t seed, uint32_t *ids,
                            float *dists) {
  return ss_search_scatter_batch_stats(h, queries, nq, K, L, num_threads, early_termination, seed,
                                       ids, dists, nullptr, nullptr, nullptr, nullptr);
}

int ss_search_scatter_batch_stats(ss_index *h, const float *queries, uint32_t nq, int K, int L,
                                  int num_threads, int early_termination, uint64_t seed,
                                  uint32_t *ids, float *dists, uint32_t *ndc_sum,
                                  uint32_t *ndc_max, uint32_t *ndc_min, uint32_t *hops_sum) {
  int rc = check_scatter_args(h, K, L, num_threads);
  if (rc) return rc;
  if (nq == 0) return SS_OK;
  if (!queries || !ids) return set_err(h, SS_ERR_INVALID_ARGUMENT, "null queries or ids");
  DeviceGuard dg(h->device);
  CtxLease lease(h);
  SearchCtx *c = lease.c;
  if (!c) return set_err(h, SS_ERR_CUDA, "cannot create a stream");
  const size_t total = (size_t)nq * K;
  const bool stats = ndc_sum || ndc_max || ndc_min || hops_sum;
  SS_CUDA(h, c->q.ensure((size_t)nq * h->dim * 4), "query buffer");
  SS_CUDA(h, c->ids.ensure(total * 4), "ids buffer");
  SS_CUDA(h, c->dists.ensure(total * 4), "dists buffer");
  if (stats) {  // four counters per query: sum, max, min of evaluations, hops
    SS_CUDA(h, c->ndc.ensure((size_t)nq * 3 * 4), "counter buffer");
    SS_CUDA(h, c->hops.ensure((size_t)nq * 4), "counter buffer");
  }
  uint32_t *d_sum = stats ? c->ndc.as<uint32_t>() : nullptr;
  uint32_t *d_max = stats ? d_sum + nq : nullptr, *d_min = stats ? d_sum + 2 * (size_t)nq : nullptr;
  uint32_t *d_hops = stats ? c->hops.as<uint32_t>() : nullptr;
  SS_CUDA(h, cudaMemcpyAsync(c->q.p, queries, (size_t)nq * h->dim * 4, cudaMemcpyHostToDevice,
                             c->stream),
          "query upload");
  rc = launch_scatter(h, c, c->q.as<float>(), nq, K, L, num_threads, early_termination, seed,
                      c->ids.as<uint32_t>(), c->dists.as<float>(), d_sum, d_hops, c->stream,
                      d_max, d_min);
  if (rc) return rc;
  c->h_status.resize(nq);
  SS_CUDA(h, cudaMemcpyAsync(ids, c->ids.p, total * 4, cudaMemcpyDeviceToHost, c->stream),
          "ids download");
  if (dists)
    SS_CUDA(h, cudaMemcpyAsync(dists, c->dists.p, total * 4, cudaMemcpyDeviceToHost, c->stream),
            "dists download");
  const std::pair<uint32_t *, const uint32_t *> outs[4] = {
      {ndc_sum, d_sum}, {ndc_max, d_max}, {ndc_min, d_min}, {hops_sum, d_hops}};
  for (const auto &o : outs)
    if (o.first)
      SS_CUDA(h, cudaMemcpyAsync(o.first, o.second, (size_t)nq * 4, cudaMemcpyDeviceToHost,
                                 c->stream),
              "counter download");
  SS_CUDA(h, cudaMemcpyAsync(c->h_status.data(), c->status.p, (size_t)nq * 4,
                             cudaMemcpyDeviceToHost, c->stream),
          "status download");
  SS_CUDA(h, cudaStreamSynchronize(c->stream), "scatter search");
  return status_to_error(h, c->h_status.data(), nq);
}

int ss_search_scatter_batch_device(ss_index *h, const float *queries, uint32_t nq, int K, int L,
                                   int num_threads, int early_termination, uint64_t seed,
                                   uint32_t *ids, float *dists, uint32_t *ndc, uint32_t *hops,
                                   void *stream) {
  int rc = check_scatter_args(h, K, L, num_threads);
  if (rc) return rc;
  if (nq == 0) return SS_OK;
  if (!queries || !ids) return set_err(h, SS_ERR_INVALID_ARGUMENT, "null queries or ids");
  DeviceGuard dg(h->device);
  std::lock_guard<std::mutex> lk(h->dev_mu);
  h->dev_last_nq = nq;
  return launch_scatter(h, &h->dev_ctx, queries, nq, K, L, num_threads, early_termination, seed,
                        ids, dists, ndc, hops, static_cast<cudaStream_t>(stream));
}

int ss_batch_status(ss_index *h, uint32_t *failed_queries) {
  if (!h || !failed_queries) return fail(nullptr, SS_ERR_INVALID_ARGUMENT, "null argument");
  DeviceGuard dg(h->device);
  std::lock_guard<std::mutex> lk(h->dev_mu);
  const uint32_t nq = h->dev_last_nq;
  *failed_queries = 0;
  if (nq == 0) return SS_OK;
  std::vector<int32_t> st(nq);
  SS_CUDA(h, cudaMemcpy(st.data(), h->dev_ctx.status.p, (size_t)nq * 4, cudaMemcpyDeviceToHost),
          "status download");
  for (uint32_t i = 0; i < nq; ++i) *failed_queries += st[i] != 0;
  return SS_OK;
}

int ss_search_batch_noalloc(ss_index *h, const float *queries, uint32_t nq, int K, int L,
                            uint32_t *ids, float *dists, void *stream) {
  int rc = check_search_args(h, K, L);
  if (rc) return rc;
  if (nq > SS_NOALLOC_MAX_QUERIES)
    return set_err(h, SS_ERR_UNSUPPORTED,
                   "nq=%u exceeds SS_NOALLOC_MAX_QUERIES=%d of the allocation-free search", nq,
                   SS_NOALLOC_MAX_QUERIES);
  if (nq == 0) return SS_OK;
  if (!queries || !ids) return set_err(h, SS_ERR_INVALID_ARGUMENT, "null queries or ids");
  static_assert(SS_NOALLOC_MAX_QUERIES == ssb::kNoallocMaxQueries, "header and scratch differ");
  static_assert((size_t)SS_NOALLOC_SCRATCH_BYTES == ssb::kNoallocScratchBytes,
                "header and scratch differ");
  DeviceGuard dg(h->device);
  const cudaStream_t st = static_cast<cudaStream_t>(stream);
  ssb::GraphView g = h->view();
  int wpb = 1;
  ssb::SmemPlan plan = plan_launch(h, g, L, nq, kSmallLaunch, &wpb);
  if (ssb::warp_search_smem_bytes(plan, wpb) > 227 * 1024)
    return set_err(h, SS_ERR_UNSUPPORTED, "L=%d needs %u bytes of shared memory per query", L,
                   plan.words_per_team * 4);
  const int blocks = persistent_blocks(h, plan, wpb, nq);
  if (blocks <= 0) return set_err(h, SS_ERR_UNSUPPORTED, "search kernel cannot be resident");
  ssb::NoallocScratch sc{};
  SS_CUDA(h, ssb::noalloc_scratch(&sc), "allocation-free scratch set-up");
  ssb::BatchArgs a{};
  a.queries = queries;
  a.qstride = h->dim;
  a.nq = nq;
  a.K0 = K;
  a.L0 = L;
  a.ids = ids;
  a.dists = dists;
  a.status = sc.status;
  a.work_counter = sc.counter;
  a.max_hops = h->n + 1;
  // The scratch keeps whatever the previous call left: reset the queue head,
  // the failure counters (first failed index to 0xFFFFFFFF, counts to 0) and
  // this batch's status words.
  SS_CUDA(h, cudaMemsetAsync(sc.counter, 0, sizeof(uint32_t), st), "scratch reset");
  SS_CUDA(h, cudaMemsetAsync(sc.failed, 0xFF, sizeof(uint32_t), st), "scratch reset");
  SS_CUDA(h, cudaMemsetAsync(sc.failed + 1, 0, (ssb::kStatusKinds - 1) * sizeof(uint32_t), st),
          "scratch reset");
  SS_CUDA(h, cudaMemsetAsync(sc.status, 0, (size_t)nq * 4, st), "scratch reset");
  SS_CUDA(h, ssb::launch_warp_search(g, a, plan, wpb, blocks, st), "search launch");
  SS_CUDA(h, ssb::launch_count_failed(sc.status, nq, sc.failed, st), "status count launch");
  uint32_t failed[ssb::kStatusKinds] = {};
  SS_CUDA(h, cudaMemcpyAsync(failed, sc.failed, sizeof(failed), cudaMemcpyDeviceToHost, st),
          "status count download");
  SS_CUDA(h, cudaStreamSynchronize(st), "allocation-free search");
  // failed[0] holds the first failed index; the per-code counts follow it
  const uint32_t first = failed[0];
  failed[0] = 0;
  return first == 0xFFFFFFFFu ? SS_OK : status_counts_to_error(h, failed, first);
}

static int intra_common(ss_index *h, const float *queries, uint32_t nq, int K, int L, int W,
                        uint32_t *ids, float *dists) {
  int rc = check_search_args(h, K, L);
  if (rc) return rc;
  if (W < 1 || W > SS_MAX_INTRA_WIDTH)
    return set_err(h, SS_ERR_INVALID_ARGUMENT, "num_threads=%d outside 1..%d", W,
                   SS_MAX_INTRA_WIDTH);
  if (nq == 0) return SS_OK;
  if (!queries || !ids) return set_err(h, SS_ERR_INVALID_ARGUMENT, "null queries or ids");
  DeviceGuard dg(h->device);
  CtxLease lease(h);
  SearchCtx *c = lease.c;
  if (!c) return set_err(h, SS_ERR_CUDA, "cannot create a stream");
  const size_t total = (size_t)nq * K;
  SS_CUDA(h, c->q.ensure((size_t)nq * h->dim * 4), "query buffer");
  SS_CUDA(h, c->ids.ensure(total * 4), "ids buffer");
  SS_CUDA(h, c->dists.ensure(total * 4), "dists buffer");
  SS_CUDA(h, cudaMemcpyAsync(c->q.p, queries, (size_t)nq * h->dim * 4, cudaMemcpyHostToDevice,
                             c->stream),
          "query upload");
  rc = launch_intra(h, c, c->q.as<float>(), nq, K, L, W, c->ids.as<uint32_t>(),
                    c->dists.as<float>(), nullptr, nullptr, c->stream);
  if (rc) return rc;
  c->h_status.resize(nq);
  SS_CUDA(h, cudaMemcpyAsync(ids, c->ids.p, total * 4, cudaMemcpyDeviceToHost, c->stream),
          "ids download");
  if (dists)
    SS_CUDA(h, cudaMemcpyAsync(dists, c->dists.p, total * 4, cudaMemcpyDeviceToHost, c->stream),
            "dists download");
  SS_CUDA(h, cudaMemcpyAsync(c->h_status.data(), c->status.p, (size_t)nq * 4,
                             cudaMemcpyDeviceToHost, c->stream),
          "status download");
  SS_CUDA(h, cudaStreamSynchronize(c->stream), "intra-query search");
  return status_to_error(h, c->h_status.data(), nq);
}

int ss_search_intra(ss_index *h, const float *query, int K, int L, int num_threads, uint32_t *ids,
                    float *dists) {
  return intra_common(h, query, 1, K, L, num_threads, ids, dists);
}

int ss_search_intra_batch(ss_index *h, const float *queries, uint32_t nq, int K, int L,
                          int num_threads, uint32_t *ids, float *dists) {
  return intra_common(h, queries, nq, K, L, num_threads, ids, dists);
}

int ss_search_intra_batch_device(ss_index *h, const float *queries, uint32_t nq, int K, int L,
                                 int num_threads, uint32_t *ids, float *dists, uint32_t *ndc,
                                 uint32_t *hops, void *stream) {
  int rc = check_search_args(h, K, L);
  if (rc) return rc;
  if (num_threads < 1 || num_threads > SS_MAX_INTRA_WIDTH)
    return set_err(h, SS_ERR_INVALID_ARGUMENT, "num_threads=%d outside 1..%d", num_threads,
                   SS_MAX_INTRA_WIDTH);
  if (!queries || !ids) return set_err(h, SS_ERR_INVALID_ARGUMENT, "null queries or ids");
  DeviceGuard dg(h->device);
  std::lock_guard<std::mutex> lk(h->dev_mu);
  h->dev_last_nq = nq;
  if (nq == 0) return SS_OK;
  return launch_intra(h, &h->dev_ctx, queries, nq, K, L, num_threads, ids, dists, ndc, hops,
                      static_cast<cudaStream_t>(stream));
}

int ss_set_tuning(ss_index *h, int warps_per_block, int hash_cap, int blocks_per_sm_cap) {
  if (!h) return fail(nullptr, SS_ERR_INVALID_ARGUMENT, "null index handle");
  if (warps_per_block < 0 || warps_per_block > 8 ||
      (warps_per_block & (warps_per_block - 1)))
    return set_err(h, SS_ERR_INVALID_ARGUMENT, "warps_per_block must be 0 (auto), 1, 2, 4 or 8");
  h->warps_per_block = warps_per_block;
  h->hash_cap_override = hash_cap > 0 ? hash_cap : 0;
  h->blocks_per_sm_cap = blocks_per_sm_cap > 0 ? blocks_per_sm_cap : 0;
  return SS_OK;
}

int ss_set_stage_layout(ss_index *h, int stage_rows, int stages_per_block) {
  if (!h) return fail(nullptr, SS_ERR_INVALID_ARGUMENT, "null index handle");
  if (stage_rows < 0 || stage_rows > 32)
    return set_err(h, SS_ERR_INVALID_ARGUMENT, "stage_rows must be in [0, 32]");
  if (stages_per_block < 0 || stages_per_block > 32)
    return set_err(h, SS_ERR_INVALID_ARGUMENT, "stages_per_block must be in [0, 32]");
  h->stage_rows = stage_rows;
  h->shared_stages = stages_per_block;
  return SS_OK;
}

int ss_set_visited_marks(ss_index *h, int mode) {
  if (!h) return fail(nullptr, SS_ERR_INVALID_ARGUMENT, "null index handle");
  if (mode != SS_VISITED_MARKS_AUTO && mode != SS_VISITED_MARKS_OFF)
    return set_err(h, SS_ERR_INVALID_ARGUMENT, "unknown visited marks mode %d", mode);
  h->visited_marks = mode;
  return SS_OK;
}

int ss_set_row_copy(ss_index *h, int mode) {
  if (!h) return fail(nullptr, SS_ERR_INVALID_ARGUMENT, "null index handle");
  if (mode != SS_ROW_COPY_AUTO && mode != SS_ROW_COPY_BULK)
    return set_err(h, SS_ERR_INVALID_ARGUMENT, "unknown row copy mode %d", mode);
  h->row_copy = mode;
  return SS_OK;
}

int ss_load_fbin(const char *path, float **data, uint32_t *num, uint32_t *dim) {
  if (!path || !data || !num || !dim) return fail(nullptr, SS_ERR_INVALID_ARGUMENT, "null argument");
  FILE *f = fopen(path, "rb");
  if (!f) return fail(nullptr, SS_ERR_IO, "cannot open %s", path);
  uint32_t hdr[2];
  if (fread(hdr, 4, 2, f) != 2) {
    fclose(f);
    return fail(nullptr, SS_ERR_FORMAT, "%s: missing fbin header", path);
  }
  const size_t count = (size_t)hdr[0] * hdr[1];
  float *buf = static_cast<float *>(malloc((count + 8) * sizeof(float)));
  if (!buf) {
    fclose(f);
    return fail(nullptr, SS_ERR_OUT_OF_MEMORY, "%s: cannot allocate %zu floats", path, count);
  }
  memset(buf + count, 0, 8 * sizeof(float));
  if (fread(buf, 4, count, f) != count) {
    fclose(f);
    free(buf);
    return fail(nullptr, SS_ERR_FORMAT, "%s: file shorter than %u x %u floats", path, hdr[0],
                hdr[1]);
  }
  fclose(f);
  *data = buf;
  *num = hdr[0];
  *dim = hdr[1];
  return SS_OK;
}

int ss_load_groundtruth(const char *path, uint32_t **ids, uint32_t *nq, uint32_t *k) {
  if (!path || !ids || !nq || !k) return fail(nullptr, SS_ERR_INVALID_ARGUMENT, "null argument");
  FILE *f = fopen(path, "rb");
  if (!f) return fail(nullptr, SS_ERR_IO, "cannot open %s", path);
  uint32_t hdr[2];
  if (fread(hdr, 4, 2, f) != 2) {
    fclose(f);
    return fail(nullptr, SS_ERR_FORMAT, "%s: missing ground-truth header", path);
  }
  const size_t count = (size_t)hdr[0] * hdr[1];
  uint32_t *buf = static_cast<uint32_t *>(malloc(std::max<size_t>(count, 1) * 4));
  if (!buf) {
    fclose(f);
    return fail(nullptr, SS_ERR_OUT_OF_MEMORY, "%s: cannot allocate", path);
  }
  if (fread(buf, 4, count, f) != count) {
    fclose(f);
    free(buf);
    return fail(nullptr, SS_ERR_FORMAT, "%s: file shorter than %u x %u ids", path, hdr[0], hdr[1]);
  }
  fclose(f);
  *ids = buf;
  *nq = hdr[0];
  *k = hdr[1];
  return SS_OK;
}

}  // extern "C"
