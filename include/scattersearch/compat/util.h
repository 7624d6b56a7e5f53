// Drop-in replacement for the reference's include/util.h: the same types and
// free functions in the global namespace, so the reference's drivers compile
// unchanged against this directory.
//
//   TestResult, Neighbor       include/util.h:11-34 (same fields)
//   load_fbin, load_groundtruth  src/util.cpp:40-93, backed by
//                              libscattersearch_b200.so (ss_load_fbin,
//                              ss_load_groundtruth)
//   load_fvecs, save_results   src/util.cpp:6-38, :94-106 (same file formats)
//   InsertIntoPool             include/util.h:41-78 (same contract, below)
//
// Every include the reference header provides (<vector>, <cstring>,
// <string>) is provided here too.
#ifndef SCATTERSEARCH_COMPAT_UTIL_H
#define SCATTERSEARCH_COMPAT_UTIL_H

#include <scattersearch/annsearch.hpp>

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#ifndef LOG
#define LOG
#endif

struct TestResult {  // include/util.h:11-21
  unsigned L;
  float throughput;
  float latency;
  float recall;
  float p95_recall;
  float p99_recall;
  float dist_comps;
  float hops;
};

// One pool entry (include/util.h:23-34): ordered by distance alone.
struct Neighbor {
  unsigned id;
  float distance;
  bool unexplored;
  Neighbor() = default;
  Neighbor(unsigned id, float distance, bool unexplored)
      : id{id}, distance{distance}, unexplored(unexplored) {}
  inline bool operator<(const Neighbor &other) const { return distance < other.distance; }
};

// Sorted insert into pool[0..K) of a pool with room for K + 1 entries, with
// the contract of the reference's InsertIntoPool (include/util.h:41-78),
// which drivers that merge per-thread pools rely on:
//   * nn nearer than every entry goes to slot 0;
//   * nn farther than every entry is stored at pool[K]; returns K;
//   * otherwise nn goes before the first entry farther than it (entries at
//     nn's distance stay ahead of it), except that when the last entry is
//     exactly at nn's distance nn takes slot K - 1, ahead of that entry;
//   * returns K + 1 and leaves the pool unchanged when an entry with nn's id
//     sits between the last entry nearer than nn and nn's slot (both
//     included), i.e. nn is already there;
//   * entries from the slot on move up by one (the last one to pool[K]).
inline int InsertIntoPool(Neighbor *pool, unsigned K, Neighbor nn) {
  if (K == 0) {
    pool[0] = nn;
    return 0;
  }
  if (nn.distance < pool[0].distance) {
    std::memmove(static_cast<void *>(pool + 1), pool, K * sizeof(Neighbor));
    pool[0] = nn;
    return 0;
  }
  if (pool[K - 1].distance < nn.distance) {
    pool[K] = nn;
    return (int)K;
  }
  unsigned lo = 0, hi = K - 1;  // first entry farther than nn, else the last slot
  while (lo < hi) {
    const unsigned mid = (lo + hi) / 2;
    if (pool[mid].distance > nn.distance) hi = mid;
    else lo = mid + 1;
  }
  const unsigned slot = hi;
  for (unsigned j = slot + 1; j-- > 0;) {
    if (pool[j].id == nn.id) return (int)K + 1;
    if (pool[j].distance < nn.distance) break;
  }
  std::memmove(static_cast<void *>(pool + slot + 1), pool + slot, (K - slot) * sizeof(Neighbor));
  pool[slot] = nn;
  return (int)slot;
}

inline void load_fbin(char *filename, float *&data, unsigned &num, unsigned &dim) {
  scattersearch::load_fbin(filename, data, num, dim);
}
inline void load_groundtruth(char *filename, std::vector<std::vector<unsigned>> &groundtruth) {
  scattersearch::load_groundtruth(filename, groundtruth);
}

// .fvecs reader (src/util.cpp:6-38): records of [int32 dim][dim floats];
// `data` receives num x dim floats allocated with new[].  Exits on a file
// that cannot be opened, as the reference does.
inline void load_fvecs(char *filename, float *&data, unsigned &num, unsigned &dim) {
  std::FILE *f = std::fopen(filename, "rb");
  if (!f) {
    std::fprintf(stderr, "open file error: %s\n", filename);
    std::exit(-1);
  }
  int d = 0;
  if (std::fread(&d, 4, 1, f) != 1 || d <= 0) {
    std::fprintf(stderr, "bad .fvecs header: %s\n", filename);
    std::exit(-1);
  }
  std::fseek(f, 0, SEEK_END);
  const long bytes = std::ftell(f);
  dim = (unsigned)d;
  num = (unsigned)((size_t)bytes / ((size_t)dim + 1) / 4);
  data = new float[(size_t)num * dim];
  std::fseek(f, 0, SEEK_SET);
  for (size_t i = 0; i < num; ++i) {
    if (std::fseek(f, 4, SEEK_CUR) != 0 || std::fread(data + i * dim, 4, dim, f) != dim) {
      std::fprintf(stderr, "truncated .fvecs file: %s\n", filename);
      std::exit(-1);
    }
  }
  std::fclose(f);
}

// Appends results as CSV with the reference's header line (src/util.cpp:94-106).
inline void save_results(const std::vector<TestResult> &results, std::string filename) {
  std::FILE *f = std::fopen(filename.c_str(), "a");
  if (!f) return;
  std::fprintf(f, "L,Throughput,latency,recall,p95recall,p99recall,dist_comps,hops\n");
  for (const TestResult &r : results)
    std::fprintf(f, "%u,%g,%g,%g,%g,%g,%g,%g\n", r.L, r.throughput, r.latency, r.recall,
                 r.p95_recall, r.p99_recall, r.dist_comps, r.hops);
  std::fclose(f);
}

#endif
