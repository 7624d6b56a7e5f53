// Drop-in replacement for the reference's include/annsearch.h: puts
// ANNSearch, Metric, L2 and INNER_PRODUCT in the global namespace, backed by
// libscattersearch_b200.so.  Put this directory ahead of the reference's
// include directory (-I include/scattersearch/compat -I include).
#ifndef SCATTERSEARCH_COMPAT_ANNSEARCH_H
#define SCATTERSEARCH_COMPAT_ANNSEARCH_H

#include <scattersearch/annsearch.hpp>

#include "util.h"

using scattersearch::ANNSearch;
using scattersearch::INNER_PRODUCT;
using scattersearch::L2;
using scattersearch::Metric;

#endif
