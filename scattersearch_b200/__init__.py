"""B200-native graph ANN search with the ScatterSearch ``ANNSearch`` surface.

The compute path is libscattersearch_b200.so: hand-written sm_100a kernels
behind the C ABI in include/scattersearch.h.  This package is the Python
host mirror of the reference interface (``ANNSearch``, ``Metric``), plus the
setup tools that make inputs for it (format I/O, synthetic workloads, graph
builder).  There is no CPU fallback: search calls raise when the native
library is missing.
"""
from .annsearch import ANNSearch, Metric  # noqa: F401
from ._native import SearchError  # noqa: F401

__all__ = ["ANNSearch", "Metric", "SearchError"]
