"""The reference's own benchmark drivers, unchanged, run against the drop-in.

oracle/Makefile builds tests/search.cpp and tests/parallel_search.cpp of the
reference twice: against the reference itself (its sources, parity flags)
and against this project's compatibility headers and library
(include/scattersearch/compat, libscattersearch_b200.so).  Both binaries run
here on the same .fbin / .nsg / ground-truth files, written with the
reference's formats, and their CSV lines are compared.

  * search (SearchArraySimulation under OpenMP, tests/search.cpp:68-114):
    the recall, p95 and p99 recall and dist_comps columns must be equal.
    The reference binary runs with OMP_THREAD_LIMIT=1: its 16 threads share
    one visited bitset that each query resets (tests/search.cpp:71-80), so
    concurrent queries corrupt one another; one thread keeps it exact.  The
    drop-in keeps each search's visited set on the device and runs as
    written, 16 threads on one index.
  * parallel_search (MultiThreadSearchArraySimulationWithET, queries one at
    a time, tests/parallel_search.cpp:66-126): entry points are random and
    the reference's threads race, so the drop-in's recall must reach the
    reference's less 0.02, and its per-query distance evaluations
    (total_dist_comps, max_dist_comps) must be filled in and within a factor
    of two of the reference's (stolen entries are copied, not taken away
    from their owner, so the GPU form evaluates more).
"""
import os
import subprocess

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
DRIVERS = os.path.join(ROOT, "oracle", "_ref", "drivers")


def _bins(name):
    ref = os.path.join(DRIVERS, f"{name}_reference")
    dropin = os.path.join(DRIVERS, f"{name}_dropin")
    if not (os.path.exists(ref) and os.path.exists(dropin)):
        pytest.skip(f"{name} drivers not built (oracle/Makefile with the reference sources)")
    return ref, dropin


@pytest.fixture(scope="module")
def files(tmp_path_factory):
    """20k x 96 unit vectors (inner product, as the drivers hard-code), 500
    queries, an NSG-style graph, exact top-100 ground truth."""
    from oracle import oracle as O
    from scattersearch_b200 import datasets, graph, io
    d = tmp_path_factory.mktemp("dropin")
    X = datasets.gaussian_mixture(20_000, 96, 20, 0.3, seed=81, mix_seed=82)
    Q = datasets.gaussian_mixture(500, 96, 20, 0.3, seed=83, mix_seed=82)
    adj, ep = graph.build_graph(X, R=32, knn_k=64, device="cpu")
    gt, _ = O.bruteforce_f64(X, Q, 100, 1)
    paths = {k: str(d / f) for k, f in (("base", "base.fbin"), ("query", "query.fbin"),
                                        ("nsg", "graph.nsg"), ("gt", "gt.bin"))}
    io.write_fbin(paths["base"], X)
    io.write_fbin(paths["query"], Q)
    io.write_nsg(paths["nsg"], adj, ep)
    io.write_groundtruth(paths["gt"], gt)
    return paths


def _run(binary, args, threads_limit=None):
    env = dict(os.environ)
    if threads_limit:
        env["OMP_THREAD_LIMIT"] = str(threads_limit)
    out = subprocess.run([binary] + args, env=env, capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, (binary, out.returncode, out.stdout[-2000:], out.stderr[-2000:])
    lines = out.stdout.splitlines()
    head = next(i for i, ln in enumerate(lines) if ln.startswith("L,"))
    cols = lines[head].split(",")
    rows = [dict(zip(cols, ln.split(","))) for ln in lines[head + 1:] if ln.count(",") >= 3]
    return rows


def test_search_driver_matches_the_reference(files):
    ref, dropin = _bins("search")
    args = [files["base"], files["query"], files["nsg"], "20,50,100", "10", files["gt"], "dropin"]
    r_rows = _run(ref, args, threads_limit=1)
    d_rows = _run(dropin, args)
    assert [r["L"] for r in r_rows] == [r["L"] for r in d_rows] == ["20", "50", "100"]
    for r, d in zip(r_rows, d_rows):
        for col in ("dist_comps", "recall", "p95recall", "p99recall"):
            assert r[col] == d[col], (r["L"], col, r[col], d[col])


def test_parallel_search_driver_tracks_the_reference(files):
    ref, dropin = _bins("parallel_search")
    for T in ("4", "8"):
        args = [files["base"], files["query"], files["nsg"], "100", "10", T, files["gt"], "dropin"]
        r_rows = _run(ref, args)
        d_rows = _run(dropin, args)
        assert len(r_rows) == len(d_rows) == 1
        r, d = r_rows[0], d_rows[0]
        assert float(d["recall"]) >= float(r["recall"]) - 0.02, (T, r, d)
        for col in ("total_dist_comps", "max_dist_comps"):
            rv, dv = float(r[col]), float(d[col])
            assert rv > 0 and 0.5 * rv <= dv <= 2.0 * rv, (T, col, rv, dv)
