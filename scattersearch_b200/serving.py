"""Online serving over one index: the ss_server_* C ABI.

``Server`` wraps the library's C++ request loop (continuous batching into the
persistent search kernel, launch slots admitted by free device memory).
``poisson_arrivals`` draws the arrival times of the online benchmark
configuration (Poisson process at a given rate).
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _native

_f32p = ctypes.POINTER(ctypes.c_float)
_u32p = ctypes.POINTER(ctypes.c_uint32)
_i32p = ctypes.POINTER(ctypes.c_int32)
_f64p = ctypes.POINTER(ctypes.c_double)


def poisson_arrivals(n: int, rate_per_s: float, seed: int = 5005) -> np.ndarray:
    """Arrival times in microseconds of n requests of a Poisson process."""
    rng = np.random.default_rng(seed)
    gaps = rng.exponential(1e6 / rate_per_s, size=n)
    return np.cumsum(gaps) - gaps[0]


class Server:
    """Continuous-batching search service over an ``ANNSearch`` index."""

    def __init__(self, index, max_batch: int = 256, max_inflight: int = 4, max_pending: int = 0,
                 K_max: int = 100, L_max: int = 512, memory_fraction: float = 0.25):
        self._lib = _native.lib()
        self._index = index
        self.dim = index.dimension
        cfg = _native.ServerConfig(max_batch, max_inflight, max_pending, K_max, L_max,
                                   memory_fraction)
        self._s = ctypes.c_void_p()
        rc = self._lib.ss_server_create(index._h, ctypes.byref(cfg), ctypes.byref(self._s))
        index._check(rc)

    def close(self):
        if self._s:
            self._lib.ss_server_destroy(self._s)
            self._s = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:  # pragma: no cover - interpreter shutdown
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def submit(self, query, K: int, L: int) -> int:
        q = np.ascontiguousarray(query, dtype=np.float32).reshape(self.dim)
        t = ctypes.c_uint64()
        self._index._check(self._lib.ss_server_submit(self._s, q.ctypes.data_as(_f32p), int(K),
                                                      int(L), ctypes.byref(t)))
        return t.value

    def wait(self, ticket: int, K: int, timeout_ms: int = -1):
        ids = np.empty(K, dtype=np.uint32)
        d = np.empty(K, dtype=np.float32)
        lat = ctypes.c_double()
        self._index._check(self._lib.ss_server_wait(self._s, int(ticket), int(timeout_ms),
                                                    ids.ctypes.data_as(_u32p),
                                                    d.ctypes.data_as(_f32p), ctypes.byref(lat)))
        return ids, d, lat.value

    def replay(self, queries, Ks, Ls, arrival_us):
        """Submits request i at arrival_us[i]; returns (ids, dists, offsets,
        latencies_us), request i's results at offsets[i] .. offsets[i]+Ks[i]."""
        q = np.ascontiguousarray(queries, dtype=np.float32)
        nq = q.shape[0]
        Ks = np.ascontiguousarray(Ks, dtype=np.int32)
        Ls = np.ascontiguousarray(Ls, dtype=np.int32)
        arr = np.ascontiguousarray(arrival_us, dtype=np.float64)
        off = np.concatenate([[0], np.cumsum(Ks)[:-1]]).astype(np.int64)
        total = int(Ks.sum())
        ids = np.empty(total, dtype=np.uint32)
        d = np.empty(total, dtype=np.float32)
        lat = np.empty(nq, dtype=np.float64)
        self._index._check(self._lib.ss_server_replay(
            self._s, q.ctypes.data_as(_f32p), nq, Ks.ctypes.data_as(_i32p),
            Ls.ctypes.data_as(_i32p), arr.ctypes.data_as(_f64p), ids.ctypes.data_as(_u32p),
            d.ctypes.data_as(_f32p), lat.ctypes.data_as(_f64p)))
        return ids, d, off, lat

    def stats(self, reset: bool = False) -> dict:
        st = _native.ServerStats()
        self._index._check(self._lib.ss_server_get_stats(self._s, ctypes.byref(st), int(reset)))
        return {name: getattr(st, name) for name, _ in st._fields_}
