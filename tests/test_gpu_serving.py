"""The serving loop (ss_server_*): continuous batching into the persistent
search kernel.

Every request's ids and distance bits must equal those of the same query
searched alone with ss_search, whatever the requests it was batched or
overlapped with: in a burst (large batches), under Poisson arrivals (batches
of every size, launches overlapping on several slots), and from several
submitting threads.
"""
import threading

import numpy as np
import pytest

from conftest import load_fixture

pytestmark = pytest.mark.gpu


def _index(fx):
    from scattersearch_b200 import ANNSearch
    idx = ANNSearch(fx["base"].shape[1], fx["base"].shape[0], fx["base"], int(fx["metric"]))
    idx.SetGraph(fx["adj"], int(fx["ep"]))
    return idx


def _alone(idx, queries, Ks, Ls):
    out = []
    for q, k, l in zip(queries, Ks, Ls):
        out.append(idx.search(q, int(k), int(l)))
    return out


def _same(a, b):
    return np.array_equal(np.asarray(a, np.float32).view(np.uint32),
                          np.asarray(b, np.float32).view(np.uint32))


@pytest.mark.parametrize("name", ["search_l2_d200", "search_ip_d96"])
def test_each_result_is_the_same_alone_and_in_the_mix(name):
    from scattersearch_b200.serving import Server, poisson_arrivals
    fx = load_fixture(name)
    idx = _index(fx)
    rng = np.random.default_rng(3)
    Q = np.concatenate([fx["queries"]] * 3)
    n = len(Q)
    Ks = rng.choice(np.array([1, 10, 32], np.int32), n)
    Ls = np.maximum(Ks, rng.integers(32, 257, n)).astype(np.int32)
    alone = _alone(idx, Q, Ks, Ls)
    with Server(idx, max_batch=16, max_inflight=3, K_max=32, L_max=256) as srv:
        for arrivals in (np.zeros(n), poisson_arrivals(n, 20000.0, seed=11)):
            ids, d, off, lat = srv.replay(Q, Ks, Ls, arrivals)
            for i in range(n):
                a_ids, a_d = alone[i]
                assert np.array_equal(ids[off[i]:off[i] + Ks[i]], a_ids), (name, i)
                assert _same(d[off[i]:off[i] + Ks[i]], a_d), (name, i)
            assert (lat > 0).all()
        st = srv.stats()
        assert st["completed"] == 2 * n and st["failed"] == 0
        assert st["batches"] > 1 and st["mean_batch"] > 1.0  # the burst was batched
        assert 0 < st["p50_us"] <= st["p99_us"] <= st["p999_us"] <= st["max_us"]
    idx.close()


def test_concurrent_submitters():
    from scattersearch_b200.serving import Server
    fx = load_fixture("search_l2_d64")
    idx = _index(fx)
    Q = fx["queries"]
    alone = _alone(idx, Q, [10] * len(Q), [50] * len(Q))
    errors = []
    with Server(idx, max_batch=8, max_inflight=2, K_max=10, L_max=64) as srv:
        def worker(t):
            try:
                tickets = [(i, srv.submit(Q[i], 10, 50)) for i in range(t, len(Q), 4)]
                for i, tk in tickets:
                    ids, d, lat = srv.wait(tk, 10)
                    if not (np.array_equal(ids, alone[i][0]) and _same(d, alone[i][1])):
                        errors.append(i)
            except Exception as e:  # pragma: no cover - reported below
                errors.append(repr(e))

        th = [threading.Thread(target=worker, args=(t,)) for t in range(4)]
        for t in th:
            t.start()
        for t in th:
            t.join()
        assert not errors
        # requests beyond the configured K/L are refused at submission
        from scattersearch_b200 import SearchError
        with pytest.raises(SearchError):
            srv.submit(Q[0], 11, 50)
        with pytest.raises(SearchError):
            srv.submit(Q[0], 5, 65)
    idx.close()


def test_request_ring_fills_and_wraps():
    from scattersearch_b200 import SearchError
    from scattersearch_b200.serving import Server
    fx = load_fixture("search_ip_d96")
    idx = _index(fx)
    Q = fx["queries"]
    alone = _alone(idx, Q, [10] * len(Q), [40] * len(Q))
    with Server(idx, max_batch=4, max_inflight=2, max_pending=8, K_max=10, L_max=40) as srv:
        tickets = [srv.submit(Q[i], 10, 40) for i in range(8)]
        with pytest.raises(SearchError) as e:
            srv.submit(Q[8], 10, 40)  # eight requests held, none collected
        assert e.value.code == 9  # SS_ERR_BUSY
        for i, t in enumerate(tickets):
            ids, d, _ = srv.wait(t, 10)
            assert np.array_equal(ids, alone[i][0]) and _same(d, alone[i][1])
        with pytest.raises(SearchError):
            srv.wait(tickets[0], 10)  # already collected
        # many wraps of the 8-entry ring, results still per query
        for rnd in range(5):
            part = list(range(rnd * 8, rnd * 8 + 8))
            tk = [(i % len(Q), srv.submit(Q[i % len(Q)], 10, 40)) for i in part]
            for i, t in tk:
                ids, d, _ = srv.wait(t, 10)
                assert np.array_equal(ids, alone[i][0]) and _same(d, alone[i][1]), (rnd, i)
    idx.close()
