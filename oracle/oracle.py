"""ctypes front end for the parity oracle.  TEST INFRASTRUCTURE ONLY.

Two libraries sit behind it (both built by oracle/Makefile):

* ``_build/libss_oracle.so`` -- the project's C restatement (ss_oracle.c) of
  the reference search, in batch-merge form;
* ``_ref/libssref.so`` / ``_ref/libssref_fast.so`` -- the reference's own
  ``ANNSearch`` compiled in place from its sources (src/annsearch.cpp,
  src/distance.cpp, src/util.cpp) behind ref_harness.cpp.  The first uses
  parity flags (no fast-math, no FMA contraction), the second the reference's
  ``-Ofast`` timing flags.

The reference libraries exist only where the reference sources were present
at build time; ``have_reference()`` tells.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_ORACLE_SO = os.path.join(_HERE, "_build", "libss_oracle.so")
_REF_SO = os.path.join(_HERE, "_ref", "libssref.so")
_REF_FAST_SO = os.path.join(_HERE, "_ref", "libssref_fast.so")

L2, IP = 0, 1
NONE_ID = 0xFFFFFFFF

_c_f32p = ctypes.POINTER(ctypes.c_float)
_c_u32p = ctypes.POINTER(ctypes.c_uint32)
_c_i32p = ctypes.POINTER(ctypes.c_int32)
_c_i64p = ctypes.POINTER(ctypes.c_int64)
_c_f64p = ctypes.POINTER(ctypes.c_double)

_libs: dict[str, ctypes.CDLL] = {}


def build() -> None:
    """Builds the oracle libraries (the reference ones only if its sources exist)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def _ptr(a, t):
    return None if a is None else a.ctypes.data_as(t)


def _lib_oracle() -> ctypes.CDLL:
    if "oracle" not in _libs:
        if not os.path.exists(_ORACLE_SO):
            build()
        lib = ctypes.CDLL(_ORACLE_SO)
        lib.sso_distance.restype = ctypes.c_float
        lib.sso_distance.argtypes = [_c_f32p, _c_f32p, ctypes.c_uint, ctypes.c_int]
        lib.sso_search_batch.restype = ctypes.c_int
        lib.sso_search_batch.argtypes = [
            _c_f32p, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_int, _c_u32p, ctypes.c_uint32,
            ctypes.c_uint32, _c_f32p, ctypes.c_uint32, _c_i32p, _c_i32p, ctypes.c_int, ctypes.c_int,
            ctypes.c_int, _c_i64p, _c_u32p, _c_f32p, _c_u32p, _c_u32p, ctypes.c_int]
        lib.sso_bruteforce.restype = ctypes.c_int
        lib.sso_bruteforce.argtypes = [
            _c_f32p, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_int, _c_f32p, ctypes.c_uint32,
            ctypes.c_int, _c_u32p, _c_f32p, ctypes.c_int]
        lib.sso_bruteforce_f64.restype = ctypes.c_int
        lib.sso_bruteforce_f64.argtypes = [
            _c_f32p, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_int, _c_f32p, ctypes.c_uint32,
            ctypes.c_int, _c_u32p, _c_f64p, ctypes.c_int]
        lib.sso_scatter_plain.restype = ctypes.c_int
        lib.sso_scatter_plain.argtypes = [
            _c_f32p, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_int, _c_u32p, ctypes.c_uint32,
            _c_f32p, ctypes.c_uint32, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_uint64,
            _c_u32p, _c_u32p, ctypes.c_int]
        _libs["oracle"] = lib
    return _libs["oracle"]


def have_reference(fast: bool = False) -> bool:
    return os.path.exists(_REF_FAST_SO if fast else _REF_SO)


def _lib_ref(fast: bool = False) -> ctypes.CDLL:
    key = "ref_fast" if fast else "ref"
    if key not in _libs:
        path = _REF_FAST_SO if fast else _REF_SO
        if not os.path.exists(path):
            raise FileNotFoundError(f"reference oracle not built: {path}")
        lib = ctypes.CDLL(path)
        lib.ssref_create.restype = ctypes.c_void_p
        lib.ssref_create.argtypes = [_c_f32p, ctypes.c_uint, ctypes.c_uint, ctypes.c_int, _c_u32p,
                                     ctypes.c_uint, ctypes.c_uint]
        lib.ssref_destroy.argtypes = [ctypes.c_void_p]
        lib.ssref_load_graph.restype = ctypes.c_int
        lib.ssref_load_graph.argtypes = [ctypes.c_void_p, ctypes.c_char_p, _c_u32p, _c_u32p, _c_u32p]
        lib.ssref_export_graph.restype = ctypes.c_int
        lib.ssref_export_graph.argtypes = [ctypes.c_void_p, _c_u32p, ctypes.c_uint]
        lib.ssref_distance.restype = ctypes.c_float
        lib.ssref_distance.argtypes = [_c_f32p, _c_f32p, ctypes.c_uint, ctypes.c_int]
        lib.ssref_search_batch.restype = ctypes.c_int
        lib.ssref_search_batch.argtypes = [ctypes.c_void_p, _c_f32p, ctypes.c_uint, ctypes.c_int,
                                           ctypes.c_int, _c_u32p, ctypes.c_int]
        lib.ssref_search_et.restype = ctypes.c_int
        lib.ssref_search_et.argtypes = [ctypes.c_void_p, _c_f32p, ctypes.c_uint, ctypes.c_int,
                                        ctypes.c_int, ctypes.c_int, ctypes.c_uint, _c_u32p, _c_f64p,
                                        _c_f64p]
        lib.ssref_search_scatter.restype = ctypes.c_int
        lib.ssref_search_scatter.argtypes = [ctypes.c_void_p, _c_f32p, ctypes.c_uint, ctypes.c_int,
                                             ctypes.c_int, ctypes.c_int, ctypes.c_uint, _c_u32p,
                                             _c_f64p, _c_f64p]
        _libs[key] = lib
    return _libs[key]


def _f32(a):
    return np.ascontiguousarray(a, dtype=np.float32)


def _u32(a):
    return np.ascontiguousarray(a, dtype=np.uint32)


def distance(a, b, metric: int) -> float:
    a, b = _f32(a), _f32(b)
    return float(_lib_oracle().sso_distance(_ptr(a, _c_f32p), _ptr(b, _c_f32p), a.shape[0], metric))


def search(base, adj, ep: int, metric: int, queries, K=None, L=None, W: int = 1, Ks=None, Ls=None,
           nthreads: int | None = None):
    """Restated SearchArraySimulation (W=1) or its W-expansions-per-step form.

    Uniform (K, L) returns ids/dists shaped (nq, K); per-query Ks/Ls return
    flat arrays laid out back to back in query order.  Also returns per-query
    distance evaluations and hops."""
    base, adj, queries = _f32(base), _u32(adj), _f32(queries)
    nq = queries.shape[0]
    nthreads = nthreads or os.cpu_count() or 1
    if Ks is not None:
        Ks = np.ascontiguousarray(Ks, dtype=np.int32)
        Ls = np.ascontiguousarray(Ls, dtype=np.int32)
        off = np.zeros(nq, dtype=np.int64)
        off[1:] = np.cumsum(Ks.astype(np.int64))[:-1]
        total = int(Ks.sum())
        ids = np.zeros(total, dtype=np.uint32)
        dists = np.zeros(total, dtype=np.float32)
        k0 = l0 = 0
    else:
        off = None
        ids = np.zeros((nq, K), dtype=np.uint32)
        dists = np.zeros((nq, K), dtype=np.float32)
        k0, l0 = int(K), int(L)
    ndc = np.zeros(nq, dtype=np.uint32)
    hops = np.zeros(nq, dtype=np.uint32)
    rc = _lib_oracle().sso_search_batch(
        _ptr(base, _c_f32p), base.shape[0], base.shape[1], metric, _ptr(adj, _c_u32p), adj.shape[1],
        int(ep), _ptr(queries, _c_f32p), nq, _ptr(Ks, _c_i32p), _ptr(Ls, _c_i32p), k0, l0, int(W),
        _ptr(off, _c_i64p), _ptr(ids, _c_u32p), _ptr(dists, _c_f32p), _ptr(ndc, _c_u32p),
        _ptr(hops, _c_u32p), int(nthreads))
    if rc != 0:
        raise ValueError("oracle search rejected its arguments")
    return ids, dists, ndc, hops


def bruteforce(base, queries, k: int, metric: int, nthreads: int | None = None):
    base, queries = _f32(base), _f32(queries)
    nq = queries.shape[0]
    ids = np.zeros((nq, k), dtype=np.uint32)
    dists = np.zeros((nq, k), dtype=np.float32)
    _lib_oracle().sso_bruteforce(_ptr(base, _c_f32p), base.shape[0], base.shape[1], metric,
                                 _ptr(queries, _c_f32p), nq, k, _ptr(ids, _c_u32p),
                                 _ptr(dists, _c_f32p), nthreads or os.cpu_count() or 1)
    return ids, dists


def bruteforce_f64(base, queries, k: int, metric: int, nthreads: int | None = None):
    """Exact k-NN with float64 distances (ties by smaller id): the ground
    truth recall is pinned against.  Returns (ids uint32, dists float64)."""
    base, queries = _f32(base), _f32(queries)
    nq = queries.shape[0]
    ids = np.zeros((nq, k), dtype=np.uint32)
    dists = np.zeros((nq, k), dtype=np.float64)
    _lib_oracle().sso_bruteforce_f64(_ptr(base, _c_f32p), base.shape[0], base.shape[1], metric,
                                     _ptr(queries, _c_f32p), nq, k, _ptr(ids, _c_u32p),
                                     _ptr(dists, _c_f64p), nthreads or os.cpu_count() or 1)
    return ids, dists


def scatter_plain(base, adj, metric: int, queries, K: int, L: int, T: int, seed: int = 1,
                  nthreads: int | None = None):
    """MultiThreadSearchArraySimulation's rules (T pools from random entry
    points, padded to L, one shared visited set, K best of all pools) under
    one fixed schedule: pools take one expansion each in turn, with an exact
    visited set.  Returns (ids nq x K, distance evaluations per query)."""
    base, adj, queries = _f32(base), _u32(adj), _f32(queries)
    nq = queries.shape[0]
    ids = np.zeros((nq, K), dtype=np.uint32)
    ndc = np.zeros(nq, dtype=np.uint32)
    rc = _lib_oracle().sso_scatter_plain(
        _ptr(base, _c_f32p), base.shape[0], base.shape[1], metric, _ptr(adj, _c_u32p),
        adj.shape[1], _ptr(queries, _c_f32p), nq, K, L, T, seed, _ptr(ids, _c_u32p),
        _ptr(ndc, _c_u32p), nthreads or os.cpu_count() or 1)
    if rc != 0:
        raise ValueError("oracle scatter search rejected its arguments")
    return ids, ndc


def recall(ids, gt, k: int = 10) -> float:
    """Mean fraction of the first k ids of each row found among gt's first k
    (the reference drivers' recall@K, tests/search.cpp:90-104)."""
    ids = np.asarray(ids)[:, :k].astype(np.int64)
    gt = np.asarray(gt)[:, :k].astype(np.int64)
    hits = sum(int(np.isin(ids[i], gt[i]).sum()) for i in range(len(ids)))
    return hits / float(k * len(ids))


def init_ties(base, adj, ep: int, queries, L: int, metric: int):
    """Per query: True when the initial pool (the first min(L, deg(ep))
    neighbours of the entry point) holds two distinct ids at exactly the same
    distance.  The reference orders that pool with std::sort, which is not
    stable (src/annsearch.cpp:215), so its order of such ties is
    implementation-defined."""
    adj = _u32(adj)
    row = adj[ep][adj[ep] != NONE_ID][:L]
    uniq = np.unique(row)
    out = np.zeros(len(queries), dtype=bool)
    if len(uniq) < 2:
        return out
    for i, q in enumerate(_f32(queries)):
        d = np.array([distance(base[j], q, metric) for j in uniq], dtype=np.float32)
        out[i] = len(np.unique(d)) != len(d)
    return out


class RefIndex:
    """The reference's ANNSearch engine, compiled in place (oracle/_ref)."""

    def __init__(self, base, metric: int, adj=None, ep: int = 0, fast: bool = False):
        self._lib = _lib_ref(fast)
        base = _f32(base)
        self.n, self.dim = base.shape
        adj_c = None if adj is None else _u32(adj)
        self._h = self._lib.ssref_create(_ptr(base, _c_f32p), self.n, self.dim, metric,
                                         _ptr(adj_c, _c_u32p), 0 if adj_c is None else adj_c.shape[1],
                                         int(ep))

    def close(self):
        if self._h:
            self._lib.ssref_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def load_graph(self, path: str):
        nodes, ep, md = ctypes.c_uint(), ctypes.c_uint(), ctypes.c_uint()
        self._lib.ssref_load_graph(self._h, path.encode(), ctypes.byref(nodes), ctypes.byref(ep),
                                   ctypes.byref(md))
        adj = np.zeros((nodes.value, max(md.value, 1)), dtype=np.uint32)
        self._lib.ssref_export_graph(self._h, _ptr(adj, _c_u32p), adj.shape[1])
        return adj, ep.value

    def search(self, queries, K: int, L: int, nthreads: int | None = None):
        queries = _f32(queries)
        ids = np.zeros((queries.shape[0], K), dtype=np.uint32)
        rc = self._lib.ssref_search_batch(self._h, _ptr(queries, _c_f32p), queries.shape[0], K, L,
                                          _ptr(ids, _c_u32p), nthreads or os.cpu_count() or 1)
        if rc != 0:
            raise ValueError("reference search rejected its arguments")
        return ids

    def search_et(self, queries, K: int, L: int, nthreads: int, seed: int = 1,
                  with_stats: bool = False):
        """MultiThreadSearchArraySimulationWithET, queries one at a time:
        (ids, per-query microseconds[, engine counters dist_comps,
        max_dist_comps, hop_count summed over the queries])."""
        queries = _f32(queries)
        ids = np.zeros((queries.shape[0], K), dtype=np.uint32)
        lat = np.zeros(queries.shape[0], dtype=np.float64)
        st = np.zeros(3, dtype=np.float64)
        rc = self._lib.ssref_search_et(self._h, _ptr(queries, _c_f32p), queries.shape[0], K, L,
                                       nthreads, seed, _ptr(ids, _c_u32p), _ptr(lat, _c_f64p),
                                       _ptr(st, _c_f64p))
        if rc != 0:
            raise ValueError("reference ET search rejected its arguments")
        return (ids, lat, st) if with_stats else (ids, lat)

    def search_scatter(self, queries, K: int, nthreads: int, seed: int = 1):
        """MultiThreadSearchArraySimulation with L = K (the only pool size its
        final merge keeps in bounds), queries one at a time: (ids, per-query
        microseconds, engine counters dist_comps, max_dist_comps, hop_count)."""
        queries = _f32(queries)
        ids = np.zeros((queries.shape[0], K), dtype=np.uint32)
        lat = np.zeros(queries.shape[0], dtype=np.float64)
        st = np.zeros(3, dtype=np.float64)
        rc = self._lib.ssref_search_scatter(self._h, _ptr(queries, _c_f32p), queries.shape[0], K,
                                            K, nthreads, seed, _ptr(ids, _c_u32p),
                                            _ptr(lat, _c_f64p), _ptr(st, _c_f64p))
        if rc != 0:
            raise ValueError("reference scatter search rejected its arguments")
        return ids, lat, st


def ref_distance(a, b, metric: int) -> float:
    a, b = _f32(a), _f32(b)
    return float(_lib_ref().ssref_distance(_ptr(a, _c_f32p), _ptr(b, _c_f32p), a.shape[0], metric))
