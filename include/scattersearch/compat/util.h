// Drop-in replacement for the reference's include/util.h: TestResult,
// load_fbin and load_groundtruth (src/util.cpp:40-93) in the global
// namespace, the loaders backed by libscattersearch_b200.so.
#ifndef SCATTERSEARCH_COMPAT_UTIL_H
#define SCATTERSEARCH_COMPAT_UTIL_H

#include <scattersearch/annsearch.hpp>

#include <vector>

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

inline void load_fbin(char *filename, float *&data, unsigned &num, unsigned &dim) {
  scattersearch::load_fbin(filename, data, num, dim);
}
inline void load_groundtruth(char *filename, std::vector<std::vector<unsigned>> &groundtruth) {
  scattersearch::load_groundtruth(filename, groundtruth);
}

#endif
