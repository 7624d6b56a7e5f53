"""ScatterSearch's intra-query search (ss_search_scatter*): a pool per warp,
one shared visited set, entry points drawn from a seed.

As with the reference's shared bitset, which warp reaches an id first
decides where it lands, so these tests judge results by validity and recall:
every returned list must hold distinct ids with their exact distances in
ascending order, recall@K against exact brute force must be at least the
plain search's (within a small margin), and on 600 queries recall@10 must be
within 0.01 of the reference's own MultiThreadSearchArraySimulation (at
L = K) and MultiThreadSearchArraySimulationWithET at the same thread count.
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
def test_scatter_et_recall_matches_the_reference(oracle_lib, angular_600, T):
    """MultiThreadSearchArraySimulationWithET (src/annsearch.cpp:839-1025)
    against the GPU form on the same 600 queries: recall@10 within 0.01."""
    O = oracle_lib
    if not O.have_reference():
        pytest.skip("reference library not built")
    X, Q, adj, ep, gt = angular_600
    K, L = 10, 100
    ref = O.RefIndex(X, 1, adj, ep)
    ref_ids, _ = ref.search_et(Q, K, L, T, seed=11)
    ref.close()
    idx = _index(X, adj, ep, 1)
    ids, d = idx.search_scatter(Q, K, L, T, early_termination=True, seed=3)
    _check_valid(O, X, Q[:50], ids[:50], d[:50], 1)
    r_ref, r_gpu = O.recall(ref_ids, gt), O.recall(ids, gt)
    assert abs(r_gpu - r_ref) <= 0.01, (T, r_gpu, r_ref)
    idx.close()


@pytest.mark.parametrize("T", [4, 8])
def test_scatter_plain_recall_matches_the_reference(oracle_lib, angular_600, T):
    """MultiThreadSearchArraySimulation (src/annsearch.cpp:532-699), the form
    without election, at L = K = 32 (its final merge writes L entries into a
    vector of K, :651-657, so only L = K stays in bounds), against the GPU
    form on the same 600 queries: recall@10 within 0.01."""
    O = oracle_lib
    if not O.have_reference():
        pytest.skip("reference library not built")
    X, Q, adj, ep, gt = angular_600
    K = 32
    ref = O.RefIndex(X, 1, adj, ep)
    ref_ids, _, _ = ref.search_scatter(Q, K, T, seed=11)
    ref.close()
    idx = _index(X, adj, ep, 1)
    ids, d = idx.search_scatter(Q, K, K, T, early_termination=False, seed=3)
    _check_valid(O, X, Q[:50], ids[:50], d[:50], 1)
    r_ref, r_gpu = O.recall(ref_ids, gt), O.recall(ids, gt)
    assert abs(r_gpu - r_ref) <= 0.01, (T, r_gpu, r_ref)
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
