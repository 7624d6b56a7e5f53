"""Python mirror of the reference's ``ANNSearch`` (include/annsearch.h:37-84).

Method names, argument order and meaning follow the reference so that code
written against its drivers reads the same; every call goes through the C
ABI of libscattersearch_b200.so.  Differences from the reference, all on the
side of reporting errors instead of undefined behaviour:

* ``LoadGraph`` raises on a missing or malformed file (the reference ignores
  a failed open, src/annsearch.cpp:66);
* ``K > L`` raises (the reference reads past its pool);
* the caller's ``flags`` bitset is not needed -- the visited set lives on the
  GPU -- but when one is passed it is reset, as the reference does at
  src/annsearch.cpp:258, so driver code that inspects it behaves the same.
"""
from __future__ import annotations

import ctypes
import enum

import numpy as np

from . import _native

_f32p = ctypes.POINTER(ctypes.c_float)
_u32p = ctypes.POINTER(ctypes.c_uint32)
_i32p = ctypes.POINTER(ctypes.c_int32)


class Metric(enum.IntEnum):
    """enum Metric (include/annsearch.h:22-26)."""
    L2 = 0
    INNER_PRODUCT = 1


def _f32(a):
    return np.ascontiguousarray(a, dtype=np.float32)


def _ptr(a, t):
    return a.ctypes.data_as(t)


def _dptr(x):
    """Device pointer from a torch tensor, an int, or None."""
    if x is None:
        return None
    if hasattr(x, "data_ptr"):
        return ctypes.c_void_p(x.data_ptr())
    return ctypes.c_void_p(int(x)) if int(x) else None


def _out(buf, shape, dtype, name):
    """A caller's output array, checked, or a new one of ``shape``."""
    if buf is None:
        return np.empty(shape, dtype=dtype)
    n = int(np.prod(shape))
    if buf.dtype != dtype or not buf.flags.c_contiguous or buf.size < n:
        raise ValueError(f"{name} must be a C-contiguous {np.dtype(dtype).name} array of "
                         f"{n} entries")
    return buf


def _query_seed(query_id: int) -> int:
    """Seed of the scatter search's entry points for one reference query id."""
    return (int(query_id) * 0x9E3779B97F4A7C15 + 1) & 0xFFFFFFFFFFFFFFFF


def _reset_flags(flags):
    if flags is not None and hasattr(flags, "reset"):
        flags.reset()


class ANNSearch:
    """Graph ANN index resident on one GPU.

    ``ANNSearch(dim, num, base, metric)`` mirrors the reference constructor
    (src/annsearch.cpp:11-58); ``base`` is a ``num x dim`` float32 array (or
    a CUDA tensor / device pointer when ``base_on_device``) and is copied to
    the device.  ``default_ep`` is 0 until a graph is loaded, as in the
    reference (src/annsearch.cpp:57).
    """

    def __init__(self, dim: int, num: int, base, metric: Metric = Metric.L2, device: int = -1,
                 base_on_device: bool = False):
        self._lib = _native.lib()
        self._h = ctypes.c_void_p()
        self.dimension = int(dim)
        self.base_num = int(num)
        self.metric = Metric(int(metric))
        self.default_ep = 0
        self.groundtruth = None
        if base_on_device:
            rc = self._lib.ss_create_from_device(self.dimension, self.base_num, _dptr(base),
                                                 int(metric), int(device), ctypes.byref(self._h))
        else:
            b = _f32(base).reshape(self.base_num, self.dimension)
            rc = self._lib.ss_create(self.dimension, self.base_num, _ptr(b, _f32p), int(metric),
                                     int(device), ctypes.byref(self._h))
        _native.check(rc, None)

    # ------------------------------------------------------------ lifetime
    def close(self):
        if self._h:
            self._lib.ss_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def _check(self, rc):
        _native.check(rc, self._h)

    # --------------------------------------------------------------- graph
    def LoadGraph(self, filename: str) -> None:
        """ANNSearch::LoadGraph (src/annsearch.cpp:64-80)."""
        self._check(self._lib.ss_load_graph(self._h, str(filename).encode()))
        self._refresh_graph_info()

    def SetGraph(self, adj, entry_point: int) -> None:
        """Sets the graph from an ``n x R`` uint32 table padded with 0xFFFFFFFF
        (the reference's public ``graph`` / ``default_ep`` members)."""
        a = np.ascontiguousarray(adj, dtype=np.uint32)
        self._check(self._lib.ss_set_graph(self._h, _ptr(a, _u32p), a.shape[0], a.shape[1],
                                           int(entry_point)))
        self._refresh_graph_info()

    def _refresh_graph_info(self):
        n, md, ep, rs = (ctypes.c_uint32() for _ in range(4))
        self._check(self._lib.ss_graph_info(self._h, ctypes.byref(n), ctypes.byref(md),
                                            ctypes.byref(ep), ctypes.byref(rs)))
        self.default_ep = ep.value
        self.max_degree = md.value
        self.rstride = rs.value

    def graph_table(self, rstride: int | None = None) -> np.ndarray:
        """The device adjacency as an ``n x rstride`` uint32 table."""
        rs = int(rstride or self.max_degree or 1)
        out = np.empty((self.base_num, rs), dtype=np.uint32)
        self._check(self._lib.ss_get_graph(self._h, _ptr(out, _u32p), rs))
        return out

    def LoadGroundtruth(self, filename: str) -> None:
        """ANNSearch::LoadGroundtruth (src/annsearch.cpp:82-101)."""
        from .io import load_groundtruth
        self.groundtruth = load_groundtruth(filename)

    # -------------------------------------------------------------- search
    def SearchArraySimulation(self, query, query_id: int, K: int, L: int, flags=None,
                              indices=None):
        """ANNSearch::SearchArraySimulation (src/annsearch.cpp:182-259).

        Returns the K ids (uint32, ascending distance); when ``indices`` is a
        list or array it is filled in place like the reference's output
        vector."""
        ids, _ = self.search(query, K, L)
        if indices is not None:
            indices[:K] = ids.tolist() if isinstance(indices, list) else ids
        _reset_flags(flags)
        return ids

    def MultiThreadSearchArraySimulation(self, query, query_id: int, K: int, L: int,
                                         num_threads: int, flags=None, indices=None):
        """ANNSearch::MultiThreadSearchArraySimulation (src/annsearch.cpp:532-699):
        ScatterSearch's intra-query search with ``num_threads`` warps, each
        with its own random entry point and pool, one shared visited set
        (``search_scatter``).  The entry points are seeded from query_id."""
        ids, _ = self.search_scatter(query, K, L, num_threads, early_termination=False,
                                     seed=_query_seed(query_id))
        ids = ids[0]
        if indices is not None:
            indices[:K] = ids.tolist() if isinstance(indices, list) else ids
        _reset_flags(flags)
        return ids

    def MultiThreadSearchArraySimulationWithET(self, query, query_id: int, K: int, L: int,
                                               num_threads: int, flags=None, indices=None):
        """ANNSearch::MultiThreadSearchArraySimulationWithET
        (src/annsearch.cpp:839-1025): the scatter search with the election at
        the 50th expansion, early termination and stealing."""
        ids, _ = self.search_scatter(query, K, L, num_threads, early_termination=True,
                                     seed=_query_seed(query_id))
        ids = ids[0]
        if indices is not None:
            indices[:K] = ids.tolist() if isinstance(indices, list) else ids
        _reset_flags(flags)
        return ids

    # ------------------------------------------------------ numpy helpers
    def search(self, query, K: int, L: int):
        """One query, one launch (the plain per-query GPU path)."""
        q = _f32(query).reshape(-1)
        ids = np.empty(K, dtype=np.uint32)
        dists = np.empty(K, dtype=np.float32)
        self._check(self._lib.ss_search(self._h, _ptr(q, _f32p), int(K), int(L), _ptr(ids, _u32p),
                                        _ptr(dists, _f32p)))
        return ids, dists

    def search_batch(self, queries, K: int, L: int, out_ids=None, out_dists=None):
        """All queries in one persistent launch; ids/dists are ``nq x K``.
        ``out_ids`` / ``out_dists`` (C-contiguous uint32 / float32 arrays,
        e.g. views of pinned buffers) receive the results when given."""
        q = _f32(queries).reshape(-1, self.dimension)
        nq = q.shape[0]
        ids = _out(out_ids, (nq, K), np.uint32, "out_ids")
        dists = _out(out_dists, (nq, K), np.float32, "out_dists")
        self._check(self._lib.ss_search_batch(self._h, _ptr(q, _f32p), nq, int(K), int(L),
                                              _ptr(ids, _u32p), _ptr(dists, _f32p)))
        return ids, dists

    def search_batch_uneven(self, queries, Ks, Ls, out_ids=None, out_dists=None):
        """Per-query K and L; returns flat ids/dists (query i at sum(Ks[:i])).
        ``out_ids``/``out_dists`` (C-contiguous uint32/float32 of sum(Ks)
        entries, e.g. views of pinned buffers) are filled in place."""
        q = _f32(queries).reshape(-1, self.dimension)
        nq = q.shape[0]
        k = np.ascontiguousarray(Ks, dtype=np.int32)
        l = np.ascontiguousarray(Ls, dtype=np.int32)
        total = int(k.sum())
        ids = _out(out_ids, (total,), np.uint32, "out_ids")
        dists = _out(out_dists, (total,), np.float32, "out_dists")
        self._check(self._lib.ss_search_batch_uneven(self._h, _ptr(q, _f32p), nq, _ptr(k, _i32p),
                                                     _ptr(l, _i32p), _ptr(ids, _u32p),
                                                     _ptr(dists, _f32p)))
        return ids, dists

    def bruteforce(self, queries, k: int):
        """Exact k nearest base rows of each query (tensor-core candidate scan,
        exact re-rank; ties by id).  Returns (ids, dists), nq x k."""
        q = _f32(queries).reshape(-1, self.dimension)
        nq = q.shape[0]
        ids = np.empty((nq, k), dtype=np.uint32)
        dists = np.empty((nq, k), dtype=np.float32)
        self._check(self._lib.ss_bruteforce(self._h, _ptr(q, _f32p), nq, int(k), _ptr(ids, _u32p),
                                            _ptr(dists, _f32p)))
        return ids, dists

    def bruteforce_device(self, queries, nq: int, k: int, ids, dists=None, stream=None):
        self._check(self._lib.ss_bruteforce_device(
            self._h, _dptr(queries), int(nq), int(k), _dptr(ids), _dptr(dists),
            ctypes.c_void_p(int(stream)) if stream else None))

    def search_scatter(self, queries, K: int, L: int, num_threads: int,
                       early_termination: bool = False, seed: int = 1):
        """ScatterSearch's intra-query search (MultiThreadSearchArraySimulation,
        or WithET when ``early_termination``): one CTA per query, a pool per
        warp, a shared visited set.  Returns (ids, dists), nq x K."""
        q = _f32(queries).reshape(-1, self.dimension)
        nq = q.shape[0]
        ids = np.empty((nq, K), dtype=np.uint32)
        dists = np.empty((nq, K), dtype=np.float32)
        self._check(self._lib.ss_search_scatter_batch(
            self._h, _ptr(q, _f32p), nq, int(K), int(L), int(num_threads),
            int(bool(early_termination)), int(seed), _ptr(ids, _u32p), _ptr(dists, _f32p)))
        return ids, dists

    def search_scatter_stats(self, queries, K: int, L: int, num_threads: int,
                             early_termination: bool = False, seed: int = 1):
        """``search_scatter`` plus the reference engine's per-query counters:
        returns (ids, dists, counters) with counters a dict of nq-long uint32
        arrays: ``ndc_sum`` (dist_comps), ``ndc_max`` / ``ndc_min`` (one warp's
        most / fewest evaluations) and ``hops_sum`` (expansions)."""
        q = _f32(queries).reshape(-1, self.dimension)
        nq = q.shape[0]
        ids = np.empty((nq, K), dtype=np.uint32)
        dists = np.empty((nq, K), dtype=np.float32)
        cnt = {k: np.empty(nq, dtype=np.uint32) for k in ("ndc_sum", "ndc_max", "ndc_min",
                                                         "hops_sum")}
        self._check(self._lib.ss_search_scatter_batch_stats(
            self._h, _ptr(q, _f32p), nq, int(K), int(L), int(num_threads),
            int(bool(early_termination)), int(seed), _ptr(ids, _u32p), _ptr(dists, _f32p),
            *(_ptr(cnt[k], _u32p) for k in ("ndc_sum", "ndc_max", "ndc_min", "hops_sum"))))
        return ids, dists, cnt

    def search_scatter_device(self, queries, nq: int, K: int, L: int, num_threads: int, ids,
                              dists=None, early_termination: bool = False, seed: int = 1,
                              ndc=None, hops=None, stream=None):
        self._check(self._lib.ss_search_scatter_batch_device(
            self._h, _dptr(queries), int(nq), int(K), int(L), int(num_threads),
            int(bool(early_termination)), int(seed), _dptr(ids), _dptr(dists), _dptr(ndc),
            _dptr(hops), ctypes.c_void_p(int(stream)) if stream else None))

    def search_intra(self, query, K: int, L: int, num_threads: int):
        q = _f32(query).reshape(-1)
        ids = np.empty(K, dtype=np.uint32)
        dists = np.empty(K, dtype=np.float32)
        self._check(self._lib.ss_search_intra(self._h, _ptr(q, _f32p), int(K), int(L),
                                              int(num_threads), _ptr(ids, _u32p),
                                              _ptr(dists, _f32p)))
        return ids, dists

    def search_intra_batch(self, queries, K: int, L: int, num_threads: int):
        q = _f32(queries).reshape(-1, self.dimension)
        nq = q.shape[0]
        ids = np.empty((nq, K), dtype=np.uint32)
        dists = np.empty((nq, K), dtype=np.float32)
        self._check(self._lib.ss_search_intra_batch(self._h, _ptr(q, _f32p), nq, int(K), int(L),
                                                    int(num_threads), _ptr(ids, _u32p),
                                                    _ptr(dists, _f32p)))
        return ids, dists

    # ----------------------------------------------- device-pointer forms
    def search_batch_device(self, queries, nq: int, ids, dists=None, K: int = 0, L: int = 0,
                            Ks=None, Ls=None, out_off=None, L_max: int = 0, ndc=None, hops=None,
                            stream=None):
        """Enqueues a batched search on device buffers (torch tensors or raw
        pointers); returns immediately.  ``stream`` is a cudaStream_t value
        (e.g. ``torch.cuda.current_stream().cuda_stream``)."""
        self._check(self._lib.ss_search_batch_device(
            self._h, _dptr(queries), int(nq), _dptr(Ks), _dptr(Ls), _dptr(out_off), int(K), int(L),
            int(L_max), _dptr(ids), _dptr(dists), _dptr(ndc), _dptr(hops),
            ctypes.c_void_p(int(stream)) if stream else None))

    def search_intra_batch_device(self, queries, nq: int, K: int, L: int, num_threads: int, ids,
                                  dists=None, ndc=None, hops=None, stream=None):
        self._check(self._lib.ss_search_intra_batch_device(
            self._h, _dptr(queries), int(nq), int(K), int(L), int(num_threads), _dptr(ids),
            _dptr(dists), _dptr(ndc), _dptr(hops),
            ctypes.c_void_p(int(stream)) if stream else None))

    def search_batch_noalloc(self, queries, nq: int, K: int, L: int, ids, dists=None,
                             stream=None):
        """Batched search on device buffers that allocates no device memory
        (ss_search_batch_noalloc): for callers that must not call cudaMalloc.
        Its scratch is a fixed static device array shared by every call in
        the process, so overlapping calls race; returns once the search on
        ``stream`` has finished."""
        self._check(self._lib.ss_search_batch_noalloc(
            self._h, _dptr(queries), int(nq), int(K), int(L), _dptr(ids), _dptr(dists),
            ctypes.c_void_p(int(stream)) if stream else None))

    def plan_batch_device(self, queries, nq: int, K: int, L: int, ids, dists=None):
        """Captures the batched device search on these fixed buffers into a
        CUDA graph (ss_plan_create); returns a ``SearchPlan``."""
        p = ctypes.c_void_p()
        self._check(self._lib.ss_plan_create(self._h, _dptr(queries), int(nq), int(K), int(L),
                                             _dptr(ids), _dptr(dists), ctypes.byref(p)))
        return SearchPlan(self, p)

    def plan_batch_uneven_device(self, queries, nq: int, Ks, Ls, out_off, L_max: int, ids,
                                 dists=None):
        """Graph-captured batched search with per-query K/L (device arrays
        Ks, Ls, out_off); returns a ``SearchPlan``."""
        p = ctypes.c_void_p()
        self._check(self._lib.ss_plan_create_uneven(
            self._h, _dptr(queries), int(nq), _dptr(Ks), _dptr(Ls), _dptr(out_off), 0, 0,
            int(L_max), _dptr(ids), _dptr(dists), ctypes.byref(p)))
        return SearchPlan(self, p)

    def batch_status(self) -> int:
        """Failed queries of the last device batch (call after synchronising)."""
        n = ctypes.c_uint32()
        self._check(self._lib.ss_batch_status(self._h, ctypes.byref(n)))
        return n.value

    def set_tuning(self, warps_per_block: int = 0, hash_cap: int = 0, blocks_per_sm_cap: int = 0,
                   shared_stages: int = 0, stage_rows: int = 0):
        """Launch layout of the batched kernel (ss_set_tuning and
        ss_set_stage_layout); never changes results."""
        self._check(self._lib.ss_set_tuning(self._h, int(warps_per_block), int(hash_cap),
                                            int(blocks_per_sm_cap)))
        self._check(self._lib.ss_set_stage_layout(self._h, int(stage_rows), int(shared_stages)))

    ROW_COPY_AUTO = 0
    ROW_COPY_BULK = 1

    def set_row_copy(self, mode: int = 0):
        """How the batched kernel fills its row stages (ss_set_row_copy):
        ROW_COPY_AUTO, four rows per gather4 tensor copy where rows allow it,
        or ROW_COPY_BULK, one bulk copy per row; never changes results."""
        self._check(self._lib.ss_set_row_copy(self._h, int(mode)))

    VISITED_MARKS_AUTO = 0
    VISITED_MARKS_OFF = 1

    def set_visited_marks(self, mode: int = 0):
        """Visited ids of the batched kernel (ss_set_visited_marks):
        VISITED_MARKS_AUTO adds exact per-team marks in device memory to the
        shared-memory table, VISITED_MARKS_OFF keeps the table alone; never
        changes results."""
        self._check(self._lib.ss_set_visited_marks(self._h, int(mode)))


class SearchPlan:
    """A graph-captured batched search (ss_plan_*): ``launch(stream)``
    replays the recorded launch with one CUDA graph launch."""

    def __init__(self, index, handle):
        self._index = index
        self._lib = index._lib
        self._p = handle

    def launch(self, stream=None):
        self._index._check(self._lib.ss_plan_launch(
            self._p, ctypes.c_void_p(int(stream)) if stream else None))

    def failed_queries(self) -> int:
        n = ctypes.c_uint32()
        self._index._check(self._lib.ss_plan_status(self._p, ctypes.byref(n)))
        return n.value

    def close(self):
        if self._p:
            self._lib.ss_plan_destroy(self._p)
            self._p = None

    def __del__(self):
        try:
            self.close()
        except Exception:  # pragma: no cover - interpreter shutdown
            pass
