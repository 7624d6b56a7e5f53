"""Generates the golden fixtures in this directory from the REFERENCE itself.

    make -C oracle REF=<reference source tree> && python tests/golden/make_golden.py

Runs only where the reference sources were available to build
oracle/_ref/libssref.so (the reference's own ANNSearch, compiled in place with
parity flags).  The outputs are committed, so the tests that use them run
anywhere.

Each search fixture holds a small base/query set, an NSG-style graph built by
scattersearch_b200.graph, and the ids returned by the reference's
SearchArraySimulation (src/annsearch.cpp:182-259) for several (K, L).  The
reference orders exactly tied initial distances with std::sort, which is not
stable (src/annsearch.cpp:215); ``init_tie`` marks the queries whose initial
pool has such ties, where the reference's order is implementation-defined.

dist_golden.npz holds distance_l2sqr_avx / distance_ip_avx outputs
(src/distance.cpp:19-56, :115-149) for random pairs at several dimensions.
nsg_golden.npz holds a small .nsg file's bytes and the adjacency the
reference's LoadGraph (src/annsearch.cpp:64-80) parsed from them.
"""
from __future__ import annotations

import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import oracle as O  # noqa: E402
from scattersearch_b200 import graph, io  # noqa: E402

NONE = 0xFFFFFFFF


def _init_ties(base, adj, ep, queries, L, metric):
    row = adj[ep][adj[ep] != NONE][:L]
    out = np.zeros(len(queries), dtype=bool)
    for i, q in enumerate(queries):
        d = np.array([O.distance(base[j], q, metric) for j in row], dtype=np.float32)
        out[i] = len(np.unique(d)) != len(d)
    return out


def make_search_fixture(name, base, queries, metric, R, cases, knn_k=None):
    adj, ep = graph.build_graph(base, R=R, knn_k=knn_k or 2 * R, device="cpu")
    ref = O.RefIndex(base, metric, adj, ep)
    out = dict(base=base, queries=queries, adj=adj, ep=np.uint32(ep), metric=np.int32(metric))
    for K, L in cases:
        out[f"ids_K{K}_L{L}"] = ref.search(queries, K, L, nthreads=4)
        out[f"init_tie_L{L}"] = _init_ties(base, adj, ep, queries, L, metric)
    ref.close()
    np.savez_compressed(os.path.join(HERE, f"{name}.npz"), **out)
    print(name, base.shape, "ep", ep, "cases", cases)


def main():
    if not O.have_reference():
        raise SystemExit("oracle/_ref/libssref.so is missing: run "
                         "`make -C oracle REF=<reference source tree>`")
    rng = np.random.default_rng(20240601)

    # Gaussian mixture, L2, dim 64 (an even number of 8-blocks)
    means = rng.standard_normal((5, 64)).astype(np.float32)
    lab = rng.integers(0, 5, 1600)
    base = (means[lab] + 0.4 * rng.standard_normal((1600, 64))).astype(np.float32)
    lab = rng.integers(0, 5, 64)
    qs = (means[lab] + 0.4 * rng.standard_normal((64, 64))).astype(np.float32)
    make_search_fixture("search_l2_d64", base, qs, O.L2, 16, [(10, 16), (10, 50), (10, 100)])

    # integer-valued, tie heavy, inner product, dim 40 (odd number of 8-blocks:
    # the tail block is accumulated first)
    base = rng.integers(0, 4, (1500, 40)).astype(np.float32)
    qs = rng.integers(0, 4, (64, 40)).astype(np.float32)
    make_search_fixture("search_ip_d40_int", base, qs, O.IP, 24, [(10, 24), (10, 64)])

    # dim 200 (25 blocks, tail first), L2, unit-normalised mixture
    means = rng.standard_normal((4, 200)).astype(np.float32)
    lab = rng.integers(0, 4, 1000)
    base = (means[lab] + 0.3 * rng.standard_normal((1000, 200))).astype(np.float32)
    base /= np.linalg.norm(base, axis=1, keepdims=True)
    lab = rng.integers(0, 4, 64)
    qs = (means[lab] + 0.3 * rng.standard_normal((64, 200))).astype(np.float32)
    qs /= np.linalg.norm(qs, axis=1, keepdims=True)
    make_search_fixture("search_l2_d200", base, qs, O.L2, 32, [(10, 32), (10, 100)])

    # dim 96, inner product on unit vectors, R = 32, K = 20
    base = rng.standard_normal((1000, 96)).astype(np.float32)
    base /= np.linalg.norm(base, axis=1, keepdims=True)
    qs = rng.standard_normal((64, 96)).astype(np.float32)
    qs /= np.linalg.norm(qs, axis=1, keepdims=True)
    make_search_fixture("search_ip_d96", base, qs, O.IP, 32, [(20, 64)])

    # distance golden vectors
    dg = {}
    for dim in (8, 16, 40, 96, 128, 200):
        a = rng.standard_normal((32, dim)).astype(np.float32)
        b = rng.standard_normal((32, dim)).astype(np.float32)
        dg[f"a_{dim}"] = a
        dg[f"b_{dim}"] = b
        for metric in (O.L2, O.IP):
            dg[f"d_{dim}_{metric}"] = np.array([O.ref_distance(a[i], b[i], metric)
                                               for i in range(32)], dtype=np.float32)
    np.savez_compressed(os.path.join(HERE, "dist_golden.npz"), **dg)
    print("dist_golden")

    # NSG loader golden: a ragged graph with an empty row and a repeated id
    n = 40
    adj = np.full((n, 6), NONE, dtype=np.uint32)
    for i in range(n):
        k = int(rng.integers(0, 7))
        adj[i, :k] = rng.integers(0, n, k)
    adj[3, :] = NONE
    adj[5, :3] = [7, 7, 1]
    with tempfile.TemporaryDirectory() as td:
        p = os.path.join(td, "g.nsg")
        io.write_nsg(p, adj, ep=11, width=6)
        raw = np.fromfile(p, dtype=np.uint8)
        ref = O.RefIndex(np.zeros((n, 8), np.float32), O.L2)
        parsed, ep = ref.load_graph(p)
        ref.close()
    np.savez_compressed(os.path.join(HERE, "nsg_golden.npz"), raw=raw, adj=parsed,
                        ep=np.uint32(ep))
    print("nsg_golden", parsed.shape, ep)


if __name__ == "__main__":
    main()
