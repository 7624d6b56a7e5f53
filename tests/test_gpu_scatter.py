"""ScatterSearch's intra-query search (ss_search_scatter*): a pool per warp,
one shared visited set, entry points drawn from a seed.

As with the reference's shared bitset, which warp reaches an id first
decides where it lands, so these tests judge results by validity and recall:
every returned list must hold distinct ids with their exact distances in
ascending order and recall@K against exact brute force must be at least the
plain search's (within a small margin).  On 600 queries, recall@10 of the
form without election must be within 0.015 of the oracle's restatement of
its rules, and the election form must reach the reference's own
MultiThreadSearchArraySimulationWithET less 0.01 at the same thread count.
"""
import numpy as np
import pytest

from conftest import load_fixture

pytestmark = pytest.mark.gpu


def _index(base, adj, ep, metric):
    from scattersearch_b200 import ANNSearch
    idx = ANNSearch(base.shape[1], base.shape[0], base, metric)
    idx.SetGraph(adj, int(ep))
    return idx


def _recall(ids, gt):
    k = gt.shape[1]
    return float(np.mean([len(set(a[:k]) & set(b)) / k for a, b in zip(ids, gt)]))


def _check_valid(O, base, queries, ids, d, metric):
    for i in range(len(queries)):
        row = ids[i]
        assert len(set(row.tolist())) == len(row), i
        ex = np.array([O.distance(queries[i], base[j], metric) for j in row], np.float32)
        assert np.array_equal(ex.view(np.uint32), d[i].view(np.uint32)), i
        assert (np.diff(d[i]) >= 0).all(), i


@pytest.mark.parametrize("name", ["search_ip_d96", "search_l2_d200"])
@pytest.mark.parametrize("et", [False, True])
def test_scatter_results_are_valid_and_recall_holds(oracle_lib, name, et):
    O = oracle_lib
    fx = load_fixture(name)
    metric = int(fx["metric"])
    idx = _index(fx["base"], fx["adj"], fx["ep"], metric)
    K, L = 10, 64
    gt, _ = O.bruteforce(fx["base"], fx["queries"], K, metric)
    plain, _ = idx.search_batch(fx["queries"], K, L)
    r_plain = _recall(plain, gt)
    for W in (1, 4, 8):
        ids, d = idx.search_scatter(fx["queries"], K, L, W, early_termination=et, seed=7)
        _check_valid(O, fx["base"], fx["queries"], ids, d, metric)
        assert _recall(ids, gt) >= r_plain - 0.05, (name, et, W)
    idx.close()


@pytest.fixture(scope="module")
def angular_600():
    """50k x 96 unit vectors from a seeded 20-component mixture (the kind of
    data the reference's ET search is written for: its election starts from a
    distance of 1000, src/annsearch.cpp:850), 600 queries, an NSG-style
    graph with R = 32 built on the device, float64 ground truth."""
    import torch
    from oracle import oracle as O
    from scattersearch_b200 import datasets, graph
    X = datasets.gaussian_mixture(50_000, 96, 20, 0.3, seed=71, mix_seed=72)
    Q = datasets.gaussian_mixture(600, 96, 20, 0.3, seed=73, mix_seed=72)
    adj, ep = graph.build_graph(torch.from_numpy(X).cuda(), R=32, knn_k=64, device="cuda")
    gt, _ = O.bruteforce_f64(X, Q, 10, 1)
    return X, Q, adj, int(ep), gt


@pytest.mark.parametrize("T", [4, 8])
def test_scatter_et_recall_holds_against_the_reference(oracle_lib, angular_600, T):
    """MultiThreadSearchArraySimulationWithET (src/annsearch.cpp:839-1025)
    and the GPU form on the same 600 queries, K = 10, L = 100.  The
    reference's recall depends on how its threads race (0.9895 free-running,
    0.9818 with its threads on one core, where it reduces to one plain
    search), so the GPU is held one-sided: at least the reference's recall
    less 0.01, and at least the plain single search's."""
    O = oracle_lib
    if not O.have_reference():
        pytest.skip("reference library not built")
    X, Q, adj, ep, gt = angular_600
    K, L = 10, 100
    ref = O.RefIndex(X, 1, adj, ep)
    ref_ids, _ = ref.search_et(Q, K, L, T, seed=11)
    plain_ids = ref.search(Q, K, L)
    ref.close()
    idx = _index(X, adj, ep, 1)
    ids, d = idx.search_scatter(Q, K, L, T, early_termination=True, seed=3)
    _check_valid(O, X, Q[:50], ids[:50], d[:50], 1)
    r_ref, r_plain, r_gpu = O.recall(ref_ids, gt), O.recall(plain_ids, gt), O.recall(ids, gt)
    assert r_gpu >= r_ref - 0.01, (T, r_gpu, r_ref)
    assert r_gpu >= r_plain - 0.005, (T, r_gpu, r_plain)
    idx.close()


@pytest.mark.parametrize("T", [4, 8])
def test_scatter_plain_recall_matches_the_restatement(oracle_lib, angular_600, T):
    """MultiThreadSearchArraySimulation (src/annsearch.cpp:532-699), the form
    without election, at L = K = 32, against the oracle's restatement of its
    rules with an exact shared visited set (oracle.scatter_plain), on the
    same 600 queries: recall@10 within 0.015.  Both draw random entry points
    (the restatement's recall moves by about 0.003 between seeds) and the
    warps' schedule is not the restatement's round robin.  The reference's
    own threads race on a bitset without atomics, which lets several of them
    keep the region near the query: its recall is higher when its threads
    run at once (0.942 at T = 4 here) and lower on one core (0.897)."""
    O = oracle_lib
    X, Q, adj, ep, gt = angular_600
    K = 32
    o_ids, _ = O.scatter_plain(X, adj, 1, Q, K, K, T, seed=5)
    idx = _index(X, adj, ep, 1)
    ids, d = idx.search_scatter(Q, K, K, T, early_termination=False, seed=3)
    _check_valid(O, X, Q[:50], ids[:50], d[:50], 1)
    r_o, r_gpu = O.recall(o_ids, gt), O.recall(ids, gt)
    assert abs(r_gpu - r_o) <= 0.015, (T, r_gpu, r_o)
    idx.close()


def test_scatter_visited_overflow_and_limits(oracle_lib):
    from scattersearch_b200 import SearchError, graph
    O = oracle_lib
    rng = np.random.default_rng(17)
    n, dim = 20000, 64
    means = rng.standard_normal((4, dim)).astype(np.float32)
    X = (means[rng.integers(0, 4, n)] + 0.4 * rng.standard_normal((n, dim))).astype(np.float32)
    Q = (means[rng.integers(0, 4, 32)] + 0.4 * rng.standard_normal((32, dim))).astype(np.float32)
    adj, ep = graph.build_graph(X, R=32, knn_k=64, device="cpu")
    idx = _index(X, adj, ep, 0)
    for et in (False, True):
        ids, d = idx.search_scatter(Q, 20, 512, 16, early_termination=et, seed=5)
        _check_valid(O, X, Q, ids, d, 0)
    with pytest.raises(SearchError):
        idx.search_scatter(Q[:1], 10, 513, 4)
    with pytest.raises(SearchError):
        idx.search_scatter(Q[:1], 10, 64, 17)
    idx.close()
