"""The tensor-core brute-force k-NN (ss_bruteforce*).

Its ids and distance bits must equal the oracle's exact scan under the
reference's FP32 distance (ties by smaller id), including integer-valued data
full of exact ties, and its k-th distance must agree with a float64 scan to
FP32 rounding.
"""
import numpy as np
import pytest

from conftest import SEARCH_FIXTURES, load_fixture

pytestmark = pytest.mark.gpu


def _index(base, metric):
    from scattersearch_b200 import ANNSearch
    return ANNSearch(base.shape[1], base.shape[0], base, metric)


def _same_bits(a, b):
    return np.array_equal(np.asarray(a, np.float32).view(np.uint32),
                          np.asarray(b, np.float32).view(np.uint32))


def _fp64_kth(base, queries, k, metric):
    B = base.astype(np.float64)
    Q = queries.astype(np.float64)
    if metric == 0:
        D = (Q * Q).sum(1)[:, None] - 2 * Q @ B.T + (B * B).sum(1)[None, :]
    else:
        D = -(Q @ B.T)
    return np.sort(D, axis=1)[:, k - 1]


@pytest.mark.parametrize("name", SEARCH_FIXTURES)
def test_bruteforce_matches_the_exact_scan(oracle_lib, name):
    fx = load_fixture(name)
    metric = int(fx["metric"])
    idx = _index(fx["base"], metric)
    for k in (1, 10, 100):
        ids, d = idx.bruteforce(fx["queries"], k)
        o_ids, o_d = oracle_lib.bruteforce(fx["base"], fx["queries"], k, metric)
        assert np.array_equal(ids, o_ids), (name, k)
        assert _same_bits(d, o_d), (name, k)
        kth = _fp64_kth(fx["base"], fx["queries"], k, metric)
        assert np.allclose(d[:, k - 1], kth, rtol=1e-5, atol=1e-5 * np.abs(kth).max())
    idx.close()


@pytest.mark.parametrize("metric", [0, 1])
def test_bruteforce_many_splits(oracle_lib, metric):
    rng = np.random.default_rng(21 + metric)
    X = rng.standard_normal((20000, 128)).astype(np.float32)
    Q = rng.standard_normal((300, 128)).astype(np.float32)
    if metric == 1:
        X /= np.linalg.norm(X, axis=1, keepdims=True)
        Q /= np.linalg.norm(Q, axis=1, keepdims=True)
    idx = _index(X, metric)
    for k in (16, 64):
        ids, d = idx.bruteforce(Q, k)
        o_ids, o_d = oracle_lib.bruteforce(X, Q, k, metric)
        assert np.array_equal(ids, o_ids) and _same_bits(d, o_d), k
    idx.close()


def test_bruteforce_small_index_and_limits():
    from scattersearch_b200 import SearchError
    X = np.random.default_rng(4).standard_normal((7, 13)).astype(np.float32)
    idx = _index(X, 0)
    ids, d = idx.bruteforce(X[:3], 10)
    assert (ids[:, 7:] == 0xFFFFFFFF).all() and (d[:, 7:] == 0).all()
    assert (ids[:, 0] == np.arange(3)).all()  # each row is its own nearest
    with pytest.raises(SearchError):
        idx.bruteforce(X[:1], 113)
    idx.close()


def test_graph_knn_from_the_brute_force(oracle_lib):
    """graph.knn_tensor_cores: each row's k nearest other rows, exactly as the
    oracle's scan ranks them (ties by id), with the row itself dropped."""
    import torch
    from scattersearch_b200 import graph
    rng = np.random.default_rng(8)
    X = rng.standard_normal((6000, 40)).astype(np.float32)
    X[100] = X[7]  # an exact duplicate: row 100's nearest is row 7 at distance 0
    k = 24
    ids, d = graph.knn_tensor_cores(torch.from_numpy(X).cuda(), k, chunk=2048)
    ids, d = ids.cpu().numpy(), d.cpu().numpy()
    sample = np.r_[0:64, 100, 5000:5064]
    o_ids, o_d = oracle_lib.bruteforce(X, X[sample], k + 1, 0)
    for row, oi, od in zip(sample, o_ids.astype(np.int64), o_d):
        keep = oi != row
        if keep.all():
            keep[-1] = False
        assert np.array_equal(ids[row], oi[keep]), row
        assert _same_bits(d[row], od[keep]), row
    assert ids[100][0] == 7 and d[100][0] == 0.0
    adj, ep = graph.build_graph(X, R=16, knn_k=k, device="cuda", knn_backend="bruteforce")
    assert adj.shape == (6000, 16) and 0 <= ep < 6000


def test_bruteforce_from_several_threads(oracle_lib):
    """Concurrent callers on one index (each call takes its own context and
    stream) get the single-caller results, also when their first calls race
    to build the index's packed base and norms."""
    import threading
    fx = load_fixture("search_l2_d200")
    ref = _index(fx["base"], int(fx["metric"]))
    Q = fx["queries"]
    want = {k: ref.bruteforce(Q, k) for k in (8, 40, 100)}
    ref.close()
    idx = _index(fx["base"], int(fx["metric"]))  # nothing built yet
    errors = []

    def worker(k):
        try:
            for _ in range(3):
                ids, d = idx.bruteforce(Q, k)
                if not (np.array_equal(ids, want[k][0]) and _same_bits(d, want[k][1])):
                    errors.append(k)
        except Exception as e:  # pragma: no cover - reported below
            errors.append(repr(e))

    th = [threading.Thread(target=worker, args=(k,)) for k in (8, 40, 100, 40)]
    for t in th:
        t.start()
    for t in th:
        t.join()
    assert not errors
    idx.close()
