"""The largest beam width the library accepts (SS_MAX_L = 4096), in the
latency layout (a few queries) and the batch layout (a batch too large to
be resident at once in the latency layout): ids and distance bits equal the
oracle's; one more is rejected before any work."""
import numpy as np
import pytest

from conftest import load_fixture

pytestmark = pytest.mark.gpu


def test_maximum_beam_width(oracle_lib):
    from scattersearch_b200 import ANNSearch, SearchError
    fx = load_fixture("search_ip_d96")
    idx = ANNSearch(fx["base"].shape[1], fx["base"].shape[0], fx["base"], int(fx["metric"]))
    idx.SetGraph(fx["adj"], int(fx["ep"]))
    Q = fx["queries"][:16]
    K, L = 100, 4096
    o_ids, o_d, _, _ = oracle_lib.search(fx["base"], fx["adj"], int(fx["ep"]),
                                         int(fx["metric"]), Q, K, L)
    ids, d = idx.search_batch(Q, K, L)
    assert np.array_equal(ids, o_ids)
    assert np.array_equal(d.view(np.uint32), o_d.view(np.uint32))
    big = np.concatenate([Q] * 170)  # 2720 queries
    ids2, d2 = idx.search_batch(big, K, L)
    assert np.array_equal(ids2, np.tile(o_ids, (170, 1)))
    assert np.array_equal(d2.view(np.uint32), np.tile(o_d, (170, 1)).view(np.uint32))
    with pytest.raises(SearchError):
        idx.search_batch(Q[:1], 10, L + 1)
    idx.close()
