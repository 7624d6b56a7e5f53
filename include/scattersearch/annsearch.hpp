// Header-only C++ drop-in for the reference's ANNSearch (include/annsearch.h:37-84)
// over the C ABI of libscattersearch_b200.so (include/scattersearch.h).
//
// Member names, argument order and meaning follow the reference so its
// drivers compile against this class; include/scattersearch/compat/ puts the
// names in the global namespace for that purpose.  Differences:
//   * the caller's `flags` bitset is accepted as any type with reset() and
//     only reset (the reference resets it at src/annsearch.cpp:258); the
//     visited set lives on the GPU;
//   * failures print the library's message and exit(-1), the reference's
//     error behaviour for loaders (src/util.cpp:42-47) applied to every call
//     (its LoadGraph ignores a failed open, src/annsearch.cpp:66);
//   * `graph` (vector<vector<unsigned>>) is not kept on the host;
//     graph_table() copies the device adjacency out on demand;
//   * the public counters follow the reference's bookkeeping: the
//     ScatterSearch methods add their distance evaluations (dist_comps), the
//     busiest warp's evaluations (max_dist_comps), max / min over the warps
//     (ub_ratio) and, without election, the expansions (hop_count), as
//     src/annsearch.cpp:634, :683-695 and :1011-1020 do; SearchArraySimulation
//     leaves them alone, as the reference does (its increments are commented
//     out, src/annsearch.cpp:212, :237).  The updates are serialised by a
//     lock, where the reference's are plain racy increments.
#ifndef SCATTERSEARCH_ANNSEARCH_HPP
#define SCATTERSEARCH_ANNSEARCH_HPP

#include <scattersearch.h>

#include <atomic>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <mutex>
#include <vector>

namespace scattersearch {

enum Metric { L2 = SS_METRIC_L2, INNER_PRODUCT = SS_METRIC_INNER_PRODUCT };

inline void die_on_error(int rc, const ss_index *h, const char *what) {
  if (rc != SS_OK) {
    std::fprintf(stderr, "%s failed (%d): %s\n", what, rc, ss_last_error(h));
    std::exit(-1);
  }
}

// load_fbin (src/util.cpp:40-70): rows plus 8 floats of zeroed slack.
inline void load_fbin(const char *filename, float *&data, unsigned &num, unsigned &dim) {
  uint32_t n = 0, d = 0;
  die_on_error(ss_load_fbin(filename, &data, &n, &d), nullptr, "load_fbin");
  num = n;
  dim = d;
}

// load_groundtruth (src/util.cpp:72-93).
inline void load_groundtruth(const char *filename, std::vector<std::vector<unsigned>> &gt) {
  uint32_t *ids = nullptr, nq = 0, k = 0;
  die_on_error(ss_load_groundtruth(filename, &ids, &nq, &k), nullptr, "load_groundtruth");
  for (uint32_t i = 0; i < nq; ++i) gt.emplace_back(ids + (size_t)i * k, ids + (size_t)(i + 1) * k);
  ss_free(ids);
}

class ANNSearch {
 public:
  // ANNSearch(dim, num, base, metric), src/annsearch.cpp:11-58.  The rows
  // are copied to the GPU; `base` stays the caller's.
  ANNSearch(unsigned dim, unsigned num, float *base, Metric m, int device = -1)
      : dimension(dim), base_num(num), base_data(base) {
    die_on_error(ss_create(dim, num, base, (int)m, device, &handle), nullptr, "ANNSearch");
  }
  ~ANNSearch() { ss_destroy(handle); }
  ANNSearch(const ANNSearch &) = delete;
  ANNSearch &operator=(const ANNSearch &) = delete;

  // src/annsearch.cpp:64-80
  void LoadGraph(const char *filename) {
    die_on_error(ss_load_graph(handle, filename), handle, "LoadGraph");
    uint32_t ep = 0;
    ss_graph_info(handle, nullptr, nullptr, &ep, nullptr);
    default_ep = ep;
  }
  // src/annsearch.cpp:82-101
  void LoadGroundtruth(const char *filename) { load_groundtruth(filename, groundtruth); }

  // Graph from an n x rstride table padded with 0xFFFFFFFF.
  void SetGraph(const std::vector<uint32_t> &adj, unsigned rstride, unsigned ep) {
    die_on_error(ss_set_graph(handle, adj.data(), (uint32_t)base_num, rstride, ep), handle,
                 "SetGraph");
    default_ep = ep;
  }

  // src/annsearch.cpp:182-259.  `indices` must hold at least K entries.
  template <class Flags>
  void SearchArraySimulation(const float *query, unsigned /*query_id*/, int K, int L, Flags &flags,
                             std::vector<unsigned> &indices) {
    if ((int)indices.size() < K) indices.resize(K);
    die_on_error(ss_search(handle, query, K, L, reinterpret_cast<uint32_t *>(indices.data()),
                           nullptr),
                 handle, "SearchArraySimulation");
    flags.reset();
  }

  // ScatterSearch's intra-query search (src/annsearch.cpp:532-699): one warp
  // per reference thread, each with its own entry point and pool, one shared
  // visited set; entry points seeded from query_id.
  template <class Flags>
  void MultiThreadSearchArraySimulation(const float *query, unsigned query_id, int K, int L,
                                        int num_threads, Flags &flags,
                                        std::vector<unsigned> &indices) {
    scatter(query, query_id, K, L, num_threads, 0, indices, "MultiThreadSearchArraySimulation");
    flags.reset();
  }

  // With the election at the 50th expansion, early termination and stealing
  // (src/annsearch.cpp:839-1025, :1368-1455).
  template <class Flags>
  void MultiThreadSearchArraySimulationWithET(const float *query, unsigned query_id, int K, int L,
                                              int num_threads, Flags &flags,
                                              std::vector<unsigned> &indices) {
    scatter(query, query_id, K, L, num_threads, 1, indices,
            "MultiThreadSearchArraySimulationWithET");
    flags.reset();
  }

  // Batched extension: nq queries, one persistent launch.  ids: nq*K.
  void SearchBatch(const float *queries, unsigned nq, int K, int L, std::vector<unsigned> &ids,
                   std::vector<float> *dists = nullptr) {
    ids.resize((size_t)nq * K);
    if (dists) dists->resize((size_t)nq * K);
    die_on_error(ss_search_batch(handle, queries, nq, K, L,
                                 reinterpret_cast<uint32_t *>(ids.data()),
                                 dists ? dists->data() : nullptr),
                 handle, "SearchBatch");
  }

  // Batched extension with per-query K and L; query i's results start at
  // Ks[0] + ... + Ks[i-1] of ids.
  void SearchBatchUneven(const float *queries, unsigned nq, const std::vector<int32_t> &Ks,
                         const std::vector<int32_t> &Ls, std::vector<unsigned> &ids,
                         std::vector<float> *dists = nullptr) {
    size_t total = 0;
    for (unsigned i = 0; i < nq; ++i) total += (size_t)Ks[i];
    ids.resize(total);
    if (dists) dists->resize(total);
    die_on_error(ss_search_batch_uneven(handle, queries, nq, Ks.data(), Ls.data(),
                                        reinterpret_cast<uint32_t *>(ids.data()),
                                        dists ? dists->data() : nullptr),
                 handle, "SearchBatchUneven");
  }

  // Launch tuning of the batched kernel (ss_set_tuning and
  // ss_set_stage_layout; 0 = automatic).  Results never depend on it.
  void SetTuning(int warps_per_block = 0, int hash_cap = 0, int blocks_per_sm_cap = 0,
                 int shared_stages = 0, int stage_rows = 0) {
    die_on_error(ss_set_tuning(handle, warps_per_block, hash_cap, blocks_per_sm_cap), handle,
                 "SetTuning");
    die_on_error(ss_set_stage_layout(handle, stage_rows, shared_stages), handle, "SetTuning");
  }

  std::vector<uint32_t> graph_table(unsigned rstride) const {
    std::vector<uint32_t> out((size_t)base_num * rstride);
    die_on_error(ss_get_graph(handle, out.data(), rstride), handle, "graph_table");
    return out;
  }

 private:
  void scatter(const float *query, unsigned query_id, int K, int L, int num_threads, int et,
               std::vector<unsigned> &indices, const char *what) {
    if ((int)indices.size() < K) indices.resize(K);
    const uint64_t seed = (uint64_t)query_id * 0x9E3779B97F4A7C15ull + 1ull;
    uint32_t sum = 0, most = 0, fewest = 0, hops = 0;
    die_on_error(ss_search_scatter_batch_stats(handle, query, 1, K, L, num_threads, et, seed,
                                               reinterpret_cast<uint32_t *>(indices.data()),
                                               nullptr, &sum, &most, &fewest, &hops),
                 handle, what);
    std::lock_guard<std::mutex> lk(counter_mu_);
    dist_comps += sum;
    max_dist_comps += most;
    ub_ratio += fewest ? (float)most / (float)fewest : 0.f;
    if (!et) hop_count += (int)hops;  // the election form keeps no hop count
  }
  std::mutex counter_mu_;

 public:
  // Public members of the reference (include/annsearch.h:58-83); drivers
  // read and reset the counters directly.
  std::atomic<int> hop_count{0};
  float ub_ratio = 0;
  int64_t dist_comps = 0;
  int64_t max_dist_comps = 0;
  double time_expand_ = 0, time_merge_ = 0, time_seq_ = 0, time_total_ = 0;
  unsigned default_ep = 0;
  size_t dimension;
  size_t base_num;
  float *base_data;
  std::vector<std::vector<unsigned>> groundtruth;
  ss_index *handle = nullptr;
};

}  // namespace scattersearch

#endif
