"""Parity of the CUDA search path with the oracle and the reference.

Every search here goes through libscattersearch_b200.so's C ABI.  The bar is
bit-exact: identical id lists and identical float32 distance bits against the
oracle (the project's C restatement, itself pinned to the reference by
test_oracle.py), and identical ids against the reference's own golden outputs
for every query whose initial pool has no exactly tied distances.
"""
import os
import threading

import numpy as np
import pytest

from conftest import NONE_ID, SEARCH_FIXTURES, fixture_cases, load_fixture

pytestmark = pytest.mark.gpu


def _index(base, adj, ep, metric):
    from scattersearch_b200 import ANNSearch
    idx = ANNSearch(base.shape[1], base.shape[0], base, metric)
    idx.SetGraph(adj, int(ep))
    return idx


def _tile(x, n=2700):
    """Rows of x repeated to at least n: a batch too large to be resident at
    once in the latency layout, so launches take the tuned layout."""
    reps = -(-n // len(x))
    return np.concatenate([x] * reps)


def _same_bits(a, b):
    return np.array_equal(np.asarray(a, np.float32).view(np.uint32),
                          np.asarray(b, np.float32).view(np.uint32))


@pytest.mark.parametrize("name", SEARCH_FIXTURES)
def test_plain_search_matches_reference_and_oracle(oracle_lib, name):
    O = oracle_lib
    fx = load_fixture(name)
    idx = _index(fx["base"], fx["adj"], fx["ep"], int(fx["metric"]))
    for K, L in fixture_cases(fx):
        o_ids, o_d, _, _ = O.search(fx["base"], fx["adj"], int(fx["ep"]), int(fx["metric"]),
                                    fx["queries"], K, L)
        ref = fx[f"ids_K{K}_L{L}"]
        tie = fx[f"init_tie_L{L}"]
        for i, q in enumerate(fx["queries"]):
            ids, d = idx.search(q, K, L)
            assert np.array_equal(ids, o_ids[i]), (name, K, L, i)
            assert _same_bits(d, o_d[i]), (name, K, L, i)
            if not tie[i]:
                assert np.array_equal(ids, ref[i]), (name, K, L, i)
    idx.close()


@pytest.mark.parametrize("name", SEARCH_FIXTURES)
def test_batched_equals_plain(oracle_lib, name):
    O = oracle_lib
    fx = load_fixture(name)
    idx = _index(fx["base"], fx["adj"], fx["ep"], int(fx["metric"]))
    for K, L in fixture_cases(fx):
        ids, d = idx.search_batch(fx["queries"], K, L)
        o_ids, o_d, _, _ = O.search(fx["base"], fx["adj"], int(fx["ep"]), int(fx["metric"]),
                                    fx["queries"], K, L)
        assert np.array_equal(ids, o_ids)
        assert _same_bits(d, o_d)
        # launch layouts (on a batch large enough to take them): teams per
        # CTA, with a stage per team or a shared pool of fewer stages (a
        # single shared stage included), stage depths from 1 to 32 rows
        big = _tile(fx["queries"])
        reps = len(big) // len(fx["queries"])
        for wpb, stages, rows in ((1, 0, 0), (2, 0, 0), (8, 0, 0), (4, 1, 0), (8, 3, 0),
                                  (8, 6, 0), (1, 0, 12), (2, 0, 5), (4, 2, 1), (2, 0, 32)):
            idx.set_tuning(warps_per_block=wpb, shared_stages=stages, stage_rows=rows)
            ids2, d2 = idx.search_batch(big, K, L)
            assert np.array_equal(ids2, np.tile(ids, (reps, 1))), (wpb, stages, rows)
            assert _same_bits(d2, np.tile(d, (reps, 1))), (wpb, stages, rows)
        idx.set_tuning()
    idx.close()


def test_uneven_batch_equals_per_query(oracle_lib):
    O = oracle_lib
    fx = load_fixture("search_l2_d200")
    idx = _index(fx["base"], fx["adj"], fx["ep"], 0)
    rng = np.random.default_rng(11)
    nq = len(fx["queries"])
    Ks = rng.choice(np.array([1, 10, 100], np.int32), nq)
    Ls = np.maximum(Ks, rng.integers(32, 513, nq)).astype(np.int32)
    ids, d = idx.search_batch_uneven(fx["queries"], Ks, Ls)
    o_ids, o_d, _, _ = O.search(fx["base"], fx["adj"], int(fx["ep"]), 0, fx["queries"], Ks=Ks,
                                Ls=Ls)
    assert np.array_equal(ids, o_ids) and _same_bits(d, o_d)
    off = 0
    for i in range(nq):
        one, od = idx.search(fx["queries"][i], int(Ks[i]), int(Ls[i]))
        assert np.array_equal(one, ids[off:off + Ks[i]])
        off += Ks[i]
    idx.close()


@pytest.mark.parametrize("W", [1, 2, 4, 8])
def test_intra_query_matches_restatement(oracle_lib, W):
    O = oracle_lib
    fx = load_fixture("search_l2_d200")
    idx = _index(fx["base"], fx["adj"], fx["ep"], 0)
    o_ids, o_d, _, _ = O.search(fx["base"], fx["adj"], int(fx["ep"]), 0, fx["queries"], 10, 100,
                                W=W)
    ids, d = idx.search_intra_batch(fx["queries"], 10, 100, W)
    assert np.array_equal(ids, o_ids)
    assert _same_bits(d, o_d)
    one, _ = idx.search_intra(fx["queries"][0], 10, 100, W)
    assert np.array_equal(one, o_ids[0])
    if W == 1:
        plain, _ = idx.search_batch(fx["queries"], 10, 100)
        assert np.array_equal(ids, plain)
    idx.close()


def _synthetic(seed, n, dim, R, metric, clusters=8):
    from scattersearch_b200 import graph
    rng = np.random.default_rng(seed)
    means = rng.standard_normal((clusters, dim)).astype(np.float32)
    X = (means[rng.integers(0, clusters, n)] + 0.4 * rng.standard_normal((n, dim))).astype(
        np.float32)
    Q = (means[rng.integers(0, clusters, 128)] + 0.4 * rng.standard_normal((128, dim))).astype(
        np.float32)
    if metric == 1:
        X /= np.linalg.norm(X, axis=1, keepdims=True)
        Q /= np.linalg.norm(Q, axis=1, keepdims=True)
    adj, ep = graph.build_graph(X, R=R, knn_k=2 * R, device="cpu")
    return X, Q, adj, ep


@pytest.mark.parametrize("dim,R,metric", [(128, 64, 0), (96, 32, 1), (13, 16, 0), (200, 32, 1),
                                          (256, 100, 0), (1100, 16, 0), (1100, 16, 1)])
def test_synthetic_shapes(oracle_lib, dim, R, metric):
    """Generic dims (13 is not a multiple of 8, 256 has no specialisation,
    1100 rows are staged in two halves), and wide graphs (R = 64 and 100
    take two and four 32-id chunks)."""
    O = oracle_lib
    X, Q, adj, ep = _synthetic(dim + R, 4000, dim, R, metric)
    idx = _index(X, adj, ep, metric)
    for K, L in ((10, 10), (10, 64), (32, 200)):
        ids, d = idx.search_batch(Q, K, L)
        o_ids, o_d, _, _ = O.search(X, adj, ep, metric, Q, K, L)
        assert np.array_equal(ids, o_ids), (dim, R, K, L)
        assert _same_bits(d, o_d)
    idx.close()


def test_visited_spill_to_global_bitset(oracle_lib):
    """A visited table far smaller than the query's visited set: the warp
    kernel's table forgets ids (they are evaluated again) and the CTA
    kernel's overflows into its global bitset; results must not change."""
    O = oracle_lib
    X, Q, adj, ep = _synthetic(5, 20000, 64, 32, 0, clusters=4)
    idx = _index(X, adj, ep, 0)
    o_ids, o_d, ndc, _ = O.search(X, adj, ep, 0, Q, 50, 400)
    assert ndc.max() > 1024  # the smallest visited table (512 slots) must overflow
    # a batch too large for the latency layout, so the 512-slot tables run
    big = _tile(Q)
    reps = len(big) // len(Q)
    o_big_ids, o_big_d = np.tile(o_ids, (reps, 1)), np.tile(o_d, (reps, 1))
    # with the per-team visited marks (default) and without (the forgetful
    # table alone)
    for marks in (idx.VISITED_MARKS_AUTO, idx.VISITED_MARKS_OFF):
        idx.set_visited_marks(marks)
        idx.set_tuning(warps_per_block=4, hash_cap=512)
        for _ in range(2):  # second pass checks the bitsets were cleared
            ids, d = idx.search_batch(big, 50, 400)
            assert np.array_equal(ids, o_big_ids) and _same_bits(d, o_big_d), marks
        idx.set_tuning(warps_per_block=8, hash_cap=512, shared_stages=2)
        ids, d = idx.search_batch(big, 50, 400)
        assert np.array_equal(ids, o_big_ids) and _same_bits(d, o_big_d), marks
    idx.set_visited_marks()
    idx.set_tuning(warps_per_block=4, hash_cap=512)
    for W in (1, 4):
        o_w, _, _, _ = O.search(X, adj, ep, 0, Q[:16], 50, 400, W=W)
        ids, _ = idx.search_intra_batch(Q[:16], 50, 400, W)
        assert np.array_equal(ids, o_w)
    idx.close()


def _rows_repeating_across_chunks(adj, seed, repeats=8):
    """Every row rewritten to hold at least 33 ids, the last `repeats` of
    them copies of ids from its first 32 (so each row repeats ids in its
    second 32-id chunk); rows shorter than 32 are first filled up with
    random other ids."""
    rng = np.random.default_rng(seed)
    n, width = adj.shape
    out = np.full((n, max(width, 64)), NONE_ID, dtype=np.uint32)
    for i in range(n):
        nb = adj[i][adj[i] != NONE_ID]
        if len(nb) < 32:
            extra = rng.choice(n, 64, replace=False)
            extra = extra[~np.isin(extra, nb) & (extra != i)][:32 - len(nb)]
            nb = np.concatenate([nb, extra.astype(np.uint32)])
        nb = nb[:64 - repeats]
        rep = nb[rng.choice(32, repeats, replace=False)]
        row = np.concatenate([nb, rep])
        out[i, :len(row)] = row
    return out


def test_repeated_ids_across_row_chunks(oracle_lib):
    """Rows of 40-64 ids (two 32-id chunks) that repeat ids of the first
    chunk in the second, searched with a visited table small enough to forget
    ids within a hop: the second occurrence must be skipped as the
    reference's visited flags skip it (src/annsearch.cpp:229-231), never
    entering the pool twice."""
    O = oracle_lib
    X, Q, _, _ = _synthetic(64 + 77, 20000, 64, 32, 0, clusters=4)
    from scattersearch_b200 import graph
    adj0, ep = graph.build_graph(X, R=48, knn_k=96, device="cpu")
    adj = _rows_repeating_across_chunks(adj0, seed=3)
    assert ((adj != NONE_ID).sum(1) > 32).all()
    idx = _index(X, adj, ep, 0)
    big = _tile(Q)
    reps = len(big) // len(Q)
    for K, L in ((10, 100), (50, 400)):
        o_ids, o_d, ndc, _ = O.search(X, adj, ep, 0, Q, K, L)
        if L == 400:
            assert ndc.max() > 1024  # far more ids than the 512-slot table holds
        for tuning, marks in ((dict(warps_per_block=4, hash_cap=512), 0),
                              (dict(warps_per_block=4, hash_cap=512), 1),
                              (dict(hash_cap=512, stage_rows=12), 1), (dict(), 0)):
            idx.set_tuning(**tuning)
            idx.set_visited_marks(marks)
            ids, d = idx.search_batch(big, K, L)
            assert np.array_equal(ids, np.tile(o_ids, (reps, 1))), (K, L, tuning)
            assert _same_bits(d, np.tile(o_d, (reps, 1))), (K, L, tuning)
            # no query's result holds an id twice unless the oracle's does
            dup = np.array([len(set(r.tolist())) < len(r) for r in ids[:len(Q)]])
            o_dup = np.array([len(set(r.tolist())) < len(r) for r in o_ids])
            assert np.array_equal(dup, o_dup)
        idx.set_tuning()
        if O.have_reference():
            ref = O.RefIndex(X, 0, adj, ep)
            r_ids = ref.search(Q, K, L)
            ref.close()
            tie = O.init_ties(X, adj, ep, Q, L, 0)
            same = (o_ids == r_ids).all(1)
            assert same[~tie].all(), np.flatnonzero(~same & ~tie)
    idx.close()


def test_repeated_ids_within_rows(oracle_lib):
    """Rows of at most 32 ids (one chunk) where every third row repeats
    some of its ids: the index notices the repeats when the graph is set and
    keeps the in-row check, so only the first copy of an id is evaluated
    (src/annsearch.cpp:229-231); a graph without repeats skips the check
    and returns the same results for the rows it shares."""
    O = oracle_lib
    X, Q, adj0, ep = _synthetic(96 + 5, 6000, 96, 24, 1)
    rng = np.random.default_rng(17)
    adj = adj0.copy()
    for i in range(0, adj.shape[0], 3):
        d = int((adj[i] != NONE_ID).sum())
        if d >= 4:
            k = int(rng.integers(1, 4))
            src = rng.choice(d, k, replace=False)
            dst = rng.choice(np.arange(1, d), k, replace=False)
            adj[i, dst] = adj[i, src]
    assert adj.shape[1] <= 32
    assert any(len(set(r[r != NONE_ID].tolist())) < int((r != NONE_ID).sum()) for r in adj)
    big = _tile(Q)
    reps = len(big) // len(Q)
    for graph_adj in (adj, adj0):
        idx = _index(X, graph_adj, ep, 1)
        for K, L in ((10, 64), (20, 200)):
            o_ids, o_d, _, _ = O.search(X, graph_adj, ep, 1, Q, K, L)
            for tuning in (dict(), dict(hash_cap=512, stage_rows=12)):
                idx.set_tuning(**tuning)
                ids, d = idx.search_batch(big, K, L)
                assert np.array_equal(ids, np.tile(o_ids, (reps, 1))), (K, L, tuning)
                assert _same_bits(d, np.tile(o_d, (reps, 1))), (K, L, tuning)
            idx.set_tuning()
        idx.close()


def test_edge_cases(oracle_lib):
    O = oracle_lib
    rng = np.random.default_rng(9)
    X = rng.standard_normal((50, 16)).astype(np.float32)
    adj = np.full((50, 8), NONE_ID, dtype=np.uint32)
    for i in range(50):
        adj[i, :6] = rng.choice(50, 6, replace=False)
    adj[7, :4] = [7, 9, 9, 3]         # self loop and repeated id in the entry row
    adj[20, :] = NONE_ID              # a node without neighbours
    idx = _index(X, adj, 7, 0)
    for K, L in ((1, 1), (4, 4), (8, 50), (50, 50)):
        ids, d = idx.search_batch(X[:10], K, L)
        o_ids, o_d, _, _ = O.search(X, adj, 7, 0, X[:10], K, L)
        assert np.array_equal(ids, o_ids) and _same_bits(d, o_d), (K, L)
    # entry point without neighbours: nothing expands, slots hold id 0 / 0.0
    idx.SetGraph(adj, 20)
    ids, d = idx.search(X[0], 5, 10)
    assert (ids == 0).all() and (d == 0).all()
    from scattersearch_b200 import SearchError
    with pytest.raises(SearchError):
        idx.search(X[0], 11, 10)       # K > L
    with pytest.raises(SearchError):
        idx.search(X[0], 1, 5000)      # L > SS_MAX_L
    with pytest.raises(SearchError):
        idx.search_intra(X[0], 1, 10, 17)
    idx.close()


def test_graph_validation_and_loader(tmp_path):
    from scattersearch_b200 import ANNSearch, SearchError, io
    X = np.random.default_rng(1).standard_normal((40, 8)).astype(np.float32)
    idx = ANNSearch(8, 40, X, 0)
    with pytest.raises(SearchError):
        idx.search(X[0], 1, 4)         # no graph yet
    with pytest.raises(SearchError):
        idx.LoadGraph(str(tmp_path / "missing.nsg"))
    g = load_fixture("nsg_golden")
    p = tmp_path / "g.nsg"
    g["raw"].tofile(p)
    idx.LoadGraph(str(p))
    assert idx.default_ep == int(g["ep"])
    got = idx.graph_table(g["adj"].shape[1])
    assert np.array_equal(got, g["adj"])
    # truncated file
    g["raw"][:-3].tofile(tmp_path / "t.nsg")
    with pytest.raises(SearchError):
        idx.LoadGraph(str(tmp_path / "t.nsg"))
    # id out of range
    bad = g["adj"].copy()
    bad[0, 0] = 40
    io.write_nsg(str(tmp_path / "b.nsg"), bad, 0)
    with pytest.raises(SearchError):
        idx.LoadGraph(str(tmp_path / "b.nsg"))
    with pytest.raises(SearchError):
        idx.SetGraph(bad, 0)
    idx.close()


def test_device_api_matches_host_api(oracle_lib):
    import torch
    fx = load_fixture("search_ip_d96")
    idx = _index(fx["base"], fx["adj"], fx["ep"], 1)
    ids_h, d_h = idx.search_batch(fx["queries"], 20, 64)
    q = torch.as_tensor(fx["queries"]).cuda()
    nq = q.shape[0]
    ids = torch.empty((nq, 20), dtype=torch.int32, device="cuda")
    d = torch.empty((nq, 20), dtype=torch.float32, device="cuda")
    ndc = torch.empty(nq, dtype=torch.int32, device="cuda")
    hops = torch.empty(nq, dtype=torch.int32, device="cuda")
    s = torch.cuda.current_stream()
    idx.search_batch_device(q, nq, ids, d, K=20, L=64, ndc=ndc, hops=hops, stream=s.cuda_stream)
    s.synchronize()
    assert idx.batch_status() == 0
    assert np.array_equal(ids.cpu().numpy().view(np.uint32), ids_h)
    assert _same_bits(d.cpu().numpy(), d_h)
    _, _, o_ndc, o_hops = oracle_lib.search(fx["base"], fx["adj"], int(fx["ep"]), 1, fx["queries"],
                                            20, 64)
    # the traversal is the reference's hop for hop; a visited table that
    # forgot ids only adds distance evaluations
    assert np.array_equal(hops.cpu().numpy().view(np.uint32), o_hops)
    assert (ndc.cpu().numpy().view(np.uint32) >= o_ndc).all()
    # with the visited marks, a small table evaluates each id once
    idx.set_tuning(hash_cap=512)
    idx.search_batch_device(q, nq, ids, d, K=20, L=64, ndc=ndc, hops=hops, stream=s.cuda_stream)
    s.synchronize()
    assert np.array_equal(ids.cpu().numpy().view(np.uint32), ids_h)
    assert np.array_equal(ndc.cpu().numpy().view(np.uint32), o_ndc)
    # with a table large enough never to forget, the counts are the reference's
    idx.set_tuning(hash_cap=65536)
    idx.search_batch_device(q, nq, ids, d, K=20, L=64, ndc=ndc, hops=hops, stream=s.cuda_stream)
    s.synchronize()
    assert np.array_equal(ids.cpu().numpy().view(np.uint32), ids_h)
    assert np.array_equal(ndc.cpu().numpy().view(np.uint32), o_ndc)
    assert np.array_equal(hops.cpu().numpy().view(np.uint32), o_hops)
    idx.close()


def test_concurrent_callers_share_one_index(oracle_lib):
    fx = load_fixture("search_l2_d64")
    idx = _index(fx["base"], fx["adj"], fx["ep"], 0)
    o_ids, _, _, _ = oracle_lib.search(fx["base"], fx["adj"], int(fx["ep"]), 0, fx["queries"], 10,
                                       50)
    errors = []

    def worker(t):
        try:
            for i in range(t, len(fx["queries"]), 4):
                ids, _ = idx.search(fx["queries"][i], 10, 50)
                if not np.array_equal(ids, o_ids[i]):
                    errors.append(i)
        except Exception as e:  # pragma: no cover - reported below
            errors.append(repr(e))

    th = [threading.Thread(target=worker, args=(t,)) for t in range(4)]
    for t in th:
        t.start()
    for t in th:
        t.join()
    assert not errors
    idx.close()


def test_reference_style_driver_surface(oracle_lib):
    """The reference drivers' calling pattern: SearchArraySimulation with a
    caller-owned flags object and a preallocated indices vector."""
    fx = load_fixture("search_l2_d64")
    idx = _index(fx["base"], fx["adj"], fx["ep"], 0)

    class Flags:
        resets = 0

        def reset(self):
            Flags.resets += 1

    flags = Flags()
    tmp = [0] * 10
    out = idx.SearchArraySimulation(fx["queries"][0], 0, 10, 50, flags, tmp)
    assert tmp == out.tolist() and Flags.resets == 1
    # the intra-query forms are the scatter search: random entry points, so
    # only the list's shape and the flags reset are fixed
    out2 = idx.MultiThreadSearchArraySimulationWithET(fx["queries"][0], 0, 10, 50, 4, flags, tmp)
    assert len(set(out2.tolist())) == 10 and tmp == out2.tolist() and Flags.resets == 2
    out3 = idx.MultiThreadSearchArraySimulation(fx["queries"][0], 1, 10, 50, 4, flags, tmp)
    assert len(set(out3.tolist())) == 10 and Flags.resets == 3
    idx.close()


def test_graph_captured_plan_matches_direct_launch(oracle_lib):
    import torch
    fx = load_fixture("search_l2_d200")
    idx = _index(fx["base"], fx["adj"], fx["ep"], 0)
    Q = fx["queries"]
    half = len(Q) // 2
    q = torch.as_tensor(Q[:half]).cuda()
    ids = torch.empty((half, 10), dtype=torch.int32, device="cuda")
    d = torch.empty((half, 10), dtype=torch.float32, device="cuda")
    plan = idx.plan_batch_device(q, half, 10, 100, ids, d)
    s = torch.cuda.current_stream()
    for part in (Q[:half], Q[half:2 * half], Q[:half]):  # new queries in the same buffer
        q.copy_(torch.as_tensor(part))
        plan.launch(s.cuda_stream)
        s.synchronize()
        assert plan.failed_queries() == 0
        o_ids, o_d, _, _ = oracle_lib.search(fx["base"], fx["adj"], int(fx["ep"]), 0, part, 10,
                                             100)
        assert np.array_equal(ids.cpu().numpy().view(np.uint32), o_ids)
        assert _same_bits(d.cpu().numpy(), o_d)
    plan.close()
    idx.close()


def test_autotuner_keeps_results_and_caches_its_choice(oracle_lib, tmp_path):
    import torch
    from scattersearch_b200 import autotune
    fx = load_fixture("search_ip_d96")
    idx = _index(fx["base"], fx["adj"], fx["ep"], 1)
    q = torch.as_tensor(fx["queries"]).cuda()
    before, _ = idx.search_batch(fx["queries"], 10, 100)
    path = str(tmp_path / "tuning.json")
    choice = autotune.autotune(idx, q, 10, 100, reps=1, path=path)
    assert choice["warps_per_block"] in (1, 2, 4, 8) and choice["hash_cap"] >= 1024
    assert choice["visited_marks"] in (0, 1)
    n_layouts = (4 * len(autotune.STAGE_ROWS_CANDIDATES) + len(
        autotune.SHARED_CANDIDATES)) * len(autotune.hash_candidates(100))
    # every layout with visited marks, the fastest few again without
    assert len(choice["table"]) == n_layouts + min(autotune.MARKS_OFF_TOP, n_layouts)
    assert sum(r["visited_marks"] for r in choice["table"]) == min(autotune.MARKS_OFF_TOP,
                                                                   n_layouts)
    after, _ = idx.search_batch(fx["queries"], 10, 100)
    assert np.array_equal(before, after)
    idx.set_tuning()
    idx.set_visited_marks()
    assert autotune.apply(idx, 100, path=path)["hash_cap"] == choice["hash_cap"]
    again, _ = idx.search_batch(fx["queries"], 10, 100)
    assert np.array_equal(before, again)
    idx.close()


def test_graph_captured_uneven_plan(oracle_lib):
    import torch
    fx = load_fixture("search_l2_d200")
    idx = _index(fx["base"], fx["adj"], fx["ep"], 0)
    rng = np.random.default_rng(23)
    Q = fx["queries"]
    nq = len(Q)
    Ks = rng.choice(np.array([1, 10, 100], np.int32), nq)
    Ls = np.maximum(Ks, rng.integers(32, 513, nq)).astype(np.int32)
    off = np.concatenate([[0], np.cumsum(Ks)[:-1]]).astype(np.int64)
    total = int(Ks.sum())
    q = torch.as_tensor(Q).cuda()
    dK, dL, doff = (torch.as_tensor(x).cuda() for x in (Ks, Ls, off))
    ids = torch.empty(total, dtype=torch.int32, device="cuda")
    d = torch.empty(total, dtype=torch.float32, device="cuda")
    # the autotuner over the uneven batch keeps the ids
    from scattersearch_b200 import autotune
    choice = autotune.autotune(idx, q, total, 512, reps=1, path=None, Ks=dK, Ls=dL,
                               out_off=doff, wpb_candidates=(2, 8), hash_caps=(1024, 4096),
                               shared_candidates=((8, 3),), stage_rows_candidates=(16,),
                               marks_off_top=2)
    assert len(choice["table"]) == 8
    plan = idx.plan_batch_uneven_device(q, nq, dK, dL, doff, 512, ids, d)
    o_ids, o_d, _, _ = oracle_lib.search(fx["base"], fx["adj"], int(fx["ep"]), 0, Q, Ks=Ks, Ls=Ls)
    s = torch.cuda.current_stream()
    for _ in range(2):
        plan.launch(s.cuda_stream)
        s.synchronize()
        assert plan.failed_queries() == 0
        assert np.array_equal(ids.cpu().numpy().view(np.uint32), o_ids)
        assert _same_bits(d.cpu().numpy(), o_d)
    plan.close()
    idx.close()


@pytest.mark.parametrize("name", ["search_l2_d200", "search_ip_d96"])
def test_small_launches_and_deep_stages_keep_results(oracle_lib, name):
    """Launches whose queries all fit on the GPU at once take the latency
    layout (32-row stages, a larger visited table); tuned layouts, 32-row
    stages among them, serve batches too large for that.  Every one returns
    the ids and distance bits of the oracle."""
    fx = load_fixture(name)
    idx = _index(fx["base"], fx["adj"], fx["ep"], int(fx["metric"]))
    Q = fx["queries"]
    K, L = 10, 100
    ids, d = idx.search_batch(Q, K, L)
    o_ids, o_d, _, _ = oracle_lib.search(fx["base"], fx["adj"], int(fx["ep"]),
                                         int(fx["metric"]), Q, K, L)
    assert np.array_equal(ids, o_ids) and _same_bits(d, o_d)
    for lo, hi in ((0, 1), (3, 10), (10, 42)):
        s_ids, s_d = idx.search_batch(Q[lo:hi], K, L)
        assert np.array_equal(s_ids, ids[lo:hi]) and _same_bits(s_d, d[lo:hi]), (lo, hi)
    one, one_d = idx.search(Q[5], K, L)
    assert np.array_equal(one, ids[5]) and _same_bits(one_d, d[5])
    big = _tile(Q)
    reps = len(big) // len(Q)
    for wpb, stages, rows in ((2, 0, 32), (4, 2, 24), (1, 0, 17)):
        idx.set_tuning(warps_per_block=wpb, shared_stages=stages, stage_rows=rows)
        t_ids, t_d = idx.search_batch(big, K, L)
        assert np.array_equal(t_ids, np.tile(ids, (reps, 1))), (wpb, stages, rows)
        assert _same_bits(t_d, np.tile(d, (reps, 1))), (wpb, stages, rows)
    idx.set_tuning()
    idx.close()


@pytest.mark.parametrize("dim,metric", [(200, 1), (96, 0), (256, 0), (13, 1)])
def test_gather_and_bulk_row_copies_agree(oracle_lib, dim, metric):
    """Row stages filled four rows per gather4 tensor copy (rows of at most
    256 floats, the default) and one bulk copy per row return the same ids
    and distance bits, in private and shared stages of 12, 16, 24 and 32
    rows, and both match the oracle.  Stages of a row count that is not a
    multiple of 4 (17) take bulk copies in either mode."""
    O = oracle_lib
    X, Q, adj, ep = _synthetic(dim + 7, 4000, dim, 32, metric)
    idx = _index(X, adj, ep, metric)
    K, L = 10, 128
    o_ids, o_d, _, _ = O.search(X, adj, ep, metric, Q, K, L)
    big = _tile(Q)
    reps = len(big) // len(Q)
    for wpb, stages, rows in ((2, 0, 12), (4, 3, 16), (2, 0, 24), (4, 2, 32), (1, 0, 17)):
        idx.set_tuning(warps_per_block=wpb, shared_stages=stages, stage_rows=rows)
        for mode in (idx.ROW_COPY_AUTO, idx.ROW_COPY_BULK):
            idx.set_row_copy(mode)
            ids, d = idx.search_batch(big, K, L)
            assert np.array_equal(ids, np.tile(o_ids, (reps, 1))), (dim, wpb, stages, rows, mode)
            assert _same_bits(d, np.tile(o_d, (reps, 1))), (dim, wpb, stages, rows, mode)
    idx.set_row_copy(idx.ROW_COPY_AUTO)
    idx.set_tuning()
    # small launches take the latency layout (32-row stages)
    ids, d = idx.search_batch(Q[:20], K, L)
    assert np.array_equal(ids, o_ids[:20]) and _same_bits(d, o_d[:20])
    idx.close()


def test_visited_marks_count_each_id_once_across_epochs(oracle_lib):
    """Per-team visited marks in device memory: with a 512-slot table that
    forgets most ids, every query evaluates exactly the reference's distinct
    ids (the oracle's count), and ids and distance bits stay the oracle's.
    One team per SM and repeated launches take every team slot through more
    than 255 queries, so each slot's byte epochs wrap and its marks are
    cleared on the device; without marks the same table evaluates more."""
    import torch
    O = oracle_lib
    X, Q, adj, ep = _synthetic(11, 20000, 64, 32, 0, clusters=4)
    idx = _index(X, adj, ep, 0)
    K, L = 20, 300
    o_ids, o_d, o_ndc, o_hops = O.search(X, adj, ep, 0, Q, K, L)
    assert o_ndc.max() > 1024
    big = _tile(Q, 3000)
    reps = len(big) // len(Q)
    t_ids, t_d, t_ndc = np.tile(o_ids, (reps, 1)), np.tile(o_d, (reps, 1)), np.tile(o_ndc, reps)
    q = torch.as_tensor(big).cuda()
    nq = q.shape[0]
    ids = torch.empty((nq, K), dtype=torch.int32, device="cuda")
    d = torch.empty((nq, K), dtype=torch.float32, device="cuda")
    ndc = torch.empty(nq, dtype=torch.int32, device="cuda")
    s = torch.cuda.current_stream()
    idx.set_tuning(warps_per_block=1, hash_cap=512, blocks_per_sm_cap=1)
    per_slot = nq / torch.cuda.get_device_properties(0).multi_processor_count
    launches = int(300 / per_slot) + 2
    for it in range(launches):
        idx.search_batch_device(q, nq, ids, d, K=K, L=L, ndc=ndc, stream=s.cuda_stream)
        s.synchronize()
        assert idx.batch_status() == 0
        assert np.array_equal(ids.cpu().numpy().view(np.uint32), t_ids), it
        assert _same_bits(d.cpu().numpy(), t_d), it
        assert np.array_equal(ndc.cpu().numpy().view(np.uint32), t_ndc), it
    idx.set_visited_marks(idx.VISITED_MARKS_OFF)
    idx.search_batch_device(q, nq, ids, d, K=K, L=L, ndc=ndc, stream=s.cuda_stream)
    s.synchronize()
    assert np.array_equal(ids.cpu().numpy().view(np.uint32), t_ids)
    assert ndc.cpu().numpy().view(np.uint32).sum() > t_ndc.sum()
    idx.set_tuning()
    idx.close()
