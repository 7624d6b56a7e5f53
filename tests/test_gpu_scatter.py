"""ScatterSearch's intra-query search (ss_search_scatter*): a pool per warp,
one shared visited set, entry points drawn from a seed.

As with the reference's shared bitset, which warp reaches an id first
decides where it lands, so these tests judge results by validity and recall:
every returned list must hold distinct ids with their exact distances in
ascending order, and recall@K against exact brute force must be at least the
plain search's (within a small margin) and, with early termination, close to
the reference's own MultiThreadSearchArraySimulationWithET at the same
thread count.
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


def test_scatter_et_recall_matches_the_reference(oracle_lib):
    O = oracle_lib
    if not O.have_reference():
        pytest.skip("reference library not built")
    fx = load_fixture("search_ip_d96")  # IP: the reference's ET needs distances < 1000
    idx = _index(fx["base"], fx["adj"], fx["ep"], 1)
    K, L, T = 10, 64, 4
    gt, _ = O.bruteforce(fx["base"], fx["queries"], K, 1)
    ref = O.RefIndex(fx["base"], 1, fx["adj"], int(fx["ep"]))
    ref_ids, _ = ref.search_et(fx["queries"], K, L, T)
    r_ref = _recall(ref_ids, gt)
    ref.close()
    ids, _ = idx.search_scatter(fx["queries"], K, L, T, early_termination=True, seed=3)
    assert _recall(ids, gt) >= r_ref - 0.05
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
