// Drop-in replacement for the reference's include/annsearch.h: puts
// ANNSearch, Metric, L2, INNER_PRODUCT and CompareByFirst in the global
// namespace, backed by libscattersearch_b200.so, and brings in everything
// the reference header brings in (include/annsearch.h:4-11: <cstddef>,
// <vector>, <queue>, <iostream>, <atomic>, <map>, boost::dynamic_bitset
// and util.h), so the reference's drivers compile unchanged.  Put this
// directory ahead of the reference's include directory:
//
//   g++ -std=c++17 -fopenmp -I <repo>/include/scattersearch/compat -I <repo>/include \
//       tests/search.cpp -L <repo>/scattersearch_b200 -lscattersearch_b200
#ifndef SCATTERSEARCH_COMPAT_ANNSEARCH_H
#define SCATTERSEARCH_COMPAT_ANNSEARCH_H

#include <atomic>
#include <cstddef>
#include <iostream>
#include <map>
#include <queue>
#include <vector>

#include <boost/dynamic_bitset.hpp>
#include <scattersearch/annsearch.hpp>

#include "util.h"

using scattersearch::ANNSearch;
using scattersearch::INNER_PRODUCT;
using scattersearch::L2;
using scattersearch::Metric;

// include/annsearch.h:28-35
struct CompareByFirst {
  constexpr bool operator()(std::pair<float, unsigned> const &a,
                            std::pair<float, unsigned> const &b) const noexcept {
    return a.first < b.first;
  }
};

#endif
