// Reference-style benchmark driver over the C++ drop-in (the shape of the
// reference's tests/search.cpp:9-118): load base/query .fbin, the .nsg graph
// and the ground truth, then for each L report QPS and recall@K -- once with
// per-query SearchArraySimulation calls from several host threads (the
// reference's OpenMP pattern, each thread with its own flags), once with one
// batched launch.
//
//   search_driver data.fbin query.fbin graph.nsg L1,L2,... K gt.bin [l2|ip] [threads]
#include <scattersearch/annsearch.hpp>

#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <sstream>
#include <string>
#include <thread>
#include <vector>

namespace {

struct NoFlags {
  void reset() {}
};

double recall_at_k(const std::vector<unsigned> &res, size_t nq, int K,
                   const std::vector<std::vector<unsigned>> &gt) {
  double total = 0;
  for (size_t i = 0; i < nq; ++i) {
    int hit = 0;
    for (int j = 0; j < K; ++j)
      for (int g = 0; g < K && g < (int)gt[i].size(); ++g)
        if (res[i * K + j] == gt[i][g]) {
          ++hit;
          break;
        }
    total += (double)hit / K;
  }
  return total / (double)nq;
}

}  // namespace

int main(int argc, char **argv) {
  if (argc < 7) {
    std::fprintf(stderr,
                 "%s data_file query_file nsg_path L1,L2,... K gt_path [l2|ip] [threads]\n",
                 argv[0]);
    return 1;
  }
  float *base = nullptr, *queries = nullptr;
  unsigned n = 0, dim = 0, nq = 0, qdim = 0;
  scattersearch::load_fbin(argv[1], base, n, dim);
  scattersearch::load_fbin(argv[2], queries, nq, qdim);
  if (dim != qdim) {
    std::fprintf(stderr, "dimension mismatch\n");
    return 1;
  }
  std::vector<int> Ls;
  {
    std::stringstream ss(argv[4]);
    std::string tok;
    while (std::getline(ss, tok, ',')) Ls.push_back(std::stoi(tok));
  }
  const int K = std::atoi(argv[5]);
  const scattersearch::Metric metric =
      (argc > 7 && std::string(argv[7]) == "l2") ? scattersearch::L2 : scattersearch::INNER_PRODUCT;
  const int threads = argc > 8 ? std::atoi(argv[8]) : 16;

  scattersearch::ANNSearch engine(dim, n, base, metric);
  engine.LoadGraph(argv[3]);
  engine.LoadGroundtruth(argv[6]);
  std::printf("L,mode,QPS,recall\n");
  for (int L : Ls) {
    std::vector<unsigned> res((size_t)nq * K);
    auto t0 = std::chrono::steady_clock::now();
    std::vector<std::thread> pool;
    for (int t = 0; t < threads; ++t) {
      pool.emplace_back([&, t]() {
        NoFlags flags;
        std::vector<unsigned> tmp(K);
        for (unsigned i = t; i < nq; i += threads) {
          engine.SearchArraySimulation(queries + (size_t)i * dim, i, K, L, flags, tmp);
          for (int j = 0; j < K; ++j) res[(size_t)i * K + j] = tmp[j];
        }
      });
    }
    for (auto &th : pool) th.join();
    double s = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    std::printf("%d,plain,%.1f,%.4f\n", L, nq / s, recall_at_k(res, nq, K, engine.groundtruth));

    std::vector<unsigned> bres;
    t0 = std::chrono::steady_clock::now();
    engine.SearchBatch(queries, nq, K, L, bres);
    s = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    std::printf("%d,batched,%.1f,%.4f\n", L, nq / s, recall_at_k(bres, nq, K, engine.groundtruth));
    if (bres != res) std::printf("%d,MISMATCH between plain and batched ids\n", L);
  }
  scattersearch::die_on_error(SS_OK, nullptr, "");
  std::free(base);
  std::free(queries);
  return 0;
}
