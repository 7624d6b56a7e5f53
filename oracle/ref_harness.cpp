// C-callable harness around the UNMODIFIED reference search, compiled in place
// from the reference sources by oracle/Makefile.  TEST INFRASTRUCTURE ONLY:
// tests/, the smoke check and bench.py's CPU-baseline leg use it as the
// parity checker and as the timed CPU baseline; the product never links it.
//
// What it wraps (reference paths):
//   ANNSearch ctor / metric dispatch         src/annsearch.cpp:11-58
//   ANNSearch::LoadGraph (.nsg reader)       src/annsearch.cpp:64-80
//   ANNSearch::SearchArraySimulation         src/annsearch.cpp:182-259
//   ANNSearch::MultiThreadSearchArraySimulation        src/annsearch.cpp:532-699
//   ANNSearch::MultiThreadSearchArraySimulationWithET  src/annsearch.cpp:839-1025
//   distance_l2sqr_avx / distance_ip_avx     src/distance.cpp:19-56, 115-149
//
// One deliberate difference from the reference's own driver: every OpenMP
// thread owns its visited bitset.  tests/search.cpp:71-80 shares one bitset
// between 16 threads while each query resets it (annsearch.cpp:258), which
// corrupts concurrent queries; the race-free pattern is the reference's own
// tests/intraxinter.cpp:74-86.
#include <annsearch.h>
#include <distance.h>
#include <omp.h>

#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <new>
#include <vector>

// Every allocation made by code in this library gets 64 bytes of slack past
// its end.  MultiThreadSearchArraySimulation merges the threads' pools into
// a vector of K entries with InsertIntoPool(final_result.data(), K, nn)
// (src/annsearch.cpp:660-666), and InsertIntoPool stores a candidate worse
// than all K at addr[K] (include/util.h:52-55): one 12-byte Neighbor past the
// vector.  The slack keeps that store inside the allocation instead of
// corrupting the heap; the reference's code is unchanged.  oracle/Makefile
// links with -Bsymbolic-functions so the reference's code in this library
// binds to these definitions.  They call malloc/free directly, so memory
// allocated here and freed elsewhere (or the reverse) stays compatible.
void* operator new(std::size_t n) {
  void* p = std::malloc(n + 64);
  if (!p) throw std::bad_alloc();
  return p;
}
void* operator new[](std::size_t n) { return operator new(n); }
void operator delete(void* p) noexcept { std::free(p); }
void operator delete[](void* p) noexcept { std::free(p); }
void operator delete(void* p, std::size_t) noexcept { std::free(p); }
void operator delete[](void* p, std::size_t) noexcept { std::free(p); }

namespace {

constexpr uint32_t kNone = 0xFFFFFFFFu;

struct RefIndex {
  std::vector<float> base;  // n*dim floats + 8 floats of slack for the AVX tail read
  unsigned n = 0, dim = 0;
  ANNSearch* eng = nullptr;
};

// The AVX distance reads up to 7 floats past `dim` when dim % 8 != 0
// (distance.cpp:32-45); load_fbin allocates 8 floats of slack for it
// (util.cpp:53).  Queries get the same slack here.
std::vector<float> padded_copy(const float* src, size_t count) {
  std::vector<float> out(count + 8, 0.0f);
  for (size_t i = 0; i < count; ++i) out[i] = src[i];
  return out;
}

}  // namespace

extern "C" {

void* ssref_create(const float* base, unsigned n, unsigned dim, int metric, const uint32_t* adj,
                   unsigned rstride, unsigned ep) {
  auto* h = new RefIndex();
  h->n = n;
  h->dim = dim;
  h->base = padded_copy(base, (size_t)n * dim);
  h->eng = new ANNSearch(dim, n, h->base.data(), metric == 0 ? L2 : INNER_PRODUCT);
  if (adj) {
    h->eng->graph.assign(n, std::vector<unsigned>());
    for (unsigned i = 0; i < n; ++i) {
      const uint32_t* row = adj + (size_t)i * rstride;
      for (unsigned m = 0; m < rstride && row[m] != kNone; ++m) h->eng->graph[i].push_back(row[m]);
    }
    h->eng->default_ep = ep;
  }
  return h;
}

void ssref_destroy(void* p) {
  auto* h = static_cast<RefIndex*>(p);
  if (!h) return;
  delete h->eng;
  delete h;
}

// Reads a .nsg file with the reference's own LoadGraph and reports what it
// parsed, so the product loader can be checked against it.
int ssref_load_graph(void* p, const char* path, unsigned* nodes, unsigned* ep, unsigned* max_deg) {
  auto* h = static_cast<RefIndex*>(p);
  h->eng->graph.clear();
  h->eng->LoadGraph(path);
  *nodes = (unsigned)h->eng->graph.size();
  *ep = h->eng->default_ep;
  unsigned md = 0;
  for (auto& r : h->eng->graph) md = r.size() > md ? (unsigned)r.size() : md;
  *max_deg = md;
  return 0;
}

// Copies the parsed graph out as a padded n x rstride table (kNone padded).
int ssref_export_graph(void* p, uint32_t* adj, unsigned rstride) {
  auto* h = static_cast<RefIndex*>(p);
  for (size_t i = 0; i < h->eng->graph.size(); ++i) {
    const auto& r = h->eng->graph[i];
    if (r.size() > rstride) return -1;
    for (unsigned m = 0; m < rstride; ++m) adj[i * rstride + m] = m < r.size() ? r[m] : kNone;
  }
  return 0;
}

float ssref_distance(const float* a, const float* b, unsigned dim, int metric) {
  std::vector<float> pa = padded_copy(a, dim), pb = padded_copy(b, dim);
  return metric == 0 ? distance_l2sqr_avx(pa.data(), pb.data(), dim)
                     : distance_ip_avx(pa.data(), pb.data(), dim);
}

// SearchArraySimulation over nq queries, OpenMP across queries with one
// visited bitset per thread.  ids: nq*K.
int ssref_search_batch(void* p, const float* queries, unsigned nq, int K, int L, uint32_t* ids,
                       int nthreads) {
  auto* h = static_cast<RefIndex*>(p);
  if (K > L || K <= 0) return -1;
  std::vector<float> q = padded_copy(queries, (size_t)nq * h->dim);
  if (nthreads <= 0) nthreads = omp_get_max_threads();
#pragma omp parallel num_threads(nthreads)
  {
    boost::dynamic_bitset<> flags(h->n, 0);
    std::vector<unsigned> tmp(K);
#pragma omp for schedule(dynamic, 4)
    for (long i = 0; i < (long)nq; ++i) {
      h->eng->SearchArraySimulation(q.data() + (size_t)i * h->dim, (unsigned)i, K, L, flags, tmp);
      for (int j = 0; j < K; ++j) ids[(size_t)i * K + j] = tmp[j];
    }
  }
  return 0;
}

// MultiThreadSearchArraySimulationWithET, queries one after another with
// `nthreads` intra-query threads (the tests/parallel_search.cpp:75-86
// pattern).  Its election starts from best_dist = 1000 (annsearch.cpp:850),
// so it is only meaningful for inner product / unit-norm data; L >= K and
// every graph row non-empty are required by its indexing.  lat_us: per-query
// wall time in microseconds (may be null); stats (may be null): the engine's
// counters after the run, [0] dist_comps, [1] max_dist_comps, [2] hop_count.
int ssref_search_et(void* p, const float* queries, unsigned nq, int K, int L, int nthreads,
                    unsigned seed, uint32_t* ids, double* lat_us, double* stats) {
  auto* h = static_cast<RefIndex*>(p);
  if (K > L || K <= 0) return -1;
  std::vector<float> q = padded_copy(queries, (size_t)nq * h->dim);
  boost::dynamic_bitset<> flags(h->n, 0);
  std::vector<unsigned> tmp(K);
  srand(seed);
  h->eng->dist_comps = 0;
  h->eng->max_dist_comps = 0;
  h->eng->hop_count = 0;
  for (unsigned i = 0; i < nq; ++i) {
    double t0 = omp_get_wtime();
    h->eng->MultiThreadSearchArraySimulationWithET(q.data() + (size_t)i * h->dim, i, K, L, nthreads,
                                                   flags, tmp);
    double t1 = omp_get_wtime();
    if (lat_us) lat_us[i] = (t1 - t0) * 1e6;
    for (int j = 0; j < K; ++j) ids[(size_t)i * K + j] = tmp[j];
  }
  if (stats) {
    stats[0] = (double)h->eng->dist_comps;
    stats[1] = (double)h->eng->max_dist_comps;
    stats[2] = (double)h->eng->hop_count;
  }
  return 0;
}

// MultiThreadSearchArraySimulation (src/annsearch.cpp:532-699), the form
// without election, queries one after another with `nthreads` intra-query
// threads.  Its final merge first copies L entries into a vector of K
// (annsearch.cpp:651-657), so only L == K stays near that vector (its one
// store past the end is absorbed by the allocation slack above); other
// values are refused here.  Every thread's random padding walks forward past
// visited ids without a bound (:568-574), which the pad ids never reach in
// practice on graphs far larger than L x nthreads.  Per-query wall time in
// microseconds to lat_us (may be null); the engine's counters are summed
// into stats[0..2] = dist_comps, max_dist_comps, hop_count (may be null).
int ssref_search_scatter(void* p, const float* queries, unsigned nq, int K, int L, int nthreads,
                         unsigned seed, uint32_t* ids, double* lat_us, double* stats) {
  auto* h = static_cast<RefIndex*>(p);
  if (K <= 0 || L != K) return -1;
  std::vector<float> q = padded_copy(queries, (size_t)nq * h->dim);
  boost::dynamic_bitset<> flags(h->n, 0);
  std::vector<unsigned> tmp(K);
  srand(seed);
  h->eng->dist_comps = 0;
  h->eng->max_dist_comps = 0;
  h->eng->hop_count = 0;
  for (unsigned i = 0; i < nq; ++i) {
    double t0 = omp_get_wtime();
    h->eng->MultiThreadSearchArraySimulation(q.data() + (size_t)i * h->dim, i, K, L, nthreads,
                                             flags, tmp);
    double t1 = omp_get_wtime();
    if (lat_us) lat_us[i] = (t1 - t0) * 1e6;
    for (int j = 0; j < K; ++j) ids[(size_t)i * K + j] = tmp[j];
  }
  if (stats) {
    stats[0] = (double)h->eng->dist_comps;
    stats[1] = (double)h->eng->max_dist_comps;
    stats[2] = (double)h->eng->hop_count;
  }
  return 0;
}

}  // extern "C"
