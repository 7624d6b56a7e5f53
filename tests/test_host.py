"""Host-side pieces: file formats, synthetic workloads, graph builder and the
replica sharding used for multi-GPU runs (world size 2 over gloo on CPU)."""
import os
import socket

import numpy as np
import pytest
import torch

from conftest import NONE_ID, load_fixture


def test_fbin_groundtruth_fvecs_roundtrip(tmp_path):
    from scattersearch_b200 import io
    X = np.random.default_rng(0).standard_normal((5, 9)).astype(np.float32)
    io.write_fbin(str(tmp_path / "a.fbin"), X)
    assert np.array_equal(io.load_fbin(str(tmp_path / "a.fbin")), X)
    gt = np.arange(20, dtype=np.uint32).reshape(4, 5)
    io.write_groundtruth(str(tmp_path / "g.bin"), gt)
    assert np.array_equal(io.load_groundtruth(str(tmp_path / "g.bin")), gt)
    rows = np.concatenate([np.full((5, 1), 9, np.int32), X.view(np.int32)], axis=1)
    rows.tofile(tmp_path / "a.fvecs")
    assert np.array_equal(io.load_fvecs(str(tmp_path / "a.fvecs")), X)
    with open(tmp_path / "a.fbin", "r+b") as f:
        f.truncate(30)
    with pytest.raises(io.FormatError):
        io.load_fbin(str(tmp_path / "a.fbin"))


def test_nsg_reader_matches_reference_parse(tmp_path):
    """tests/golden/nsg_golden.npz holds a .nsg file (ragged rows, an empty
    row, a repeated id) and what the reference's LoadGraph parsed from it."""
    from scattersearch_b200 import io
    g = load_fixture("nsg_golden")
    p = tmp_path / "g.nsg"
    g["raw"].tofile(p)
    adj, ep, width = io.read_nsg(str(p))
    assert ep == int(g["ep"]) and width == 6
    ref = g["adj"]
    assert adj.shape[0] == ref.shape[0]
    R = max(adj.shape[1], ref.shape[1])
    pad = lambda a: np.pad(a, ((0, 0), (0, R - a.shape[1])), constant_values=NONE_ID)
    assert np.array_equal(pad(adj), pad(ref))
    io.write_nsg(str(tmp_path / "h.nsg"), adj, ep, width)
    assert (tmp_path / "h.nsg").read_bytes() == p.read_bytes()


def test_datasets_are_seeded_and_shaped():
    from scattersearch_b200 import datasets
    a = datasets.config(1, scale=0.01, n_queries=10)
    b = datasets.config(1, scale=0.01, n_queries=10)
    assert a.base.shape == (1000, 200) and a.queries.shape == (10, 200)
    assert np.array_equal(a.base, b.base) and np.array_equal(a.queries, b.queries)
    assert np.allclose(np.linalg.norm(a.base, axis=1), 1.0, atol=1e-5)
    c = datasets.config(2, scale=0.001, n_queries=10)
    assert c.base.shape[1] == 128 and c.base.min() >= 0 and c.base.max() <= 255
    assert np.array_equal(c.base, np.round(c.base))
    d = datasets.config(3, scale=0.001, n_queries=10)
    assert d.metric == datasets.IP and d.K == 100 and d.L_list == [200, 400]
    Ks, Ls = datasets.uneven_k_l(1000)
    assert set(np.unique(Ks)) <= {1, 10, 100} and (Ls >= Ks).all()
    assert Ls.min() >= 32 and Ls.max() <= 512


def test_graph_builder_invariants_and_recall(oracle_lib):
    from scattersearch_b200 import datasets, graph
    w = datasets.config(3, scale=0.005, n_queries=100)
    adj, ep = graph.build_graph(w.base, R=32, knn_k=64, device="cpu")
    n = w.base.shape[0]
    assert adj.shape == (n, 32) and adj.dtype == np.uint32 and 0 <= ep < n
    valid = adj != NONE_ID
    # valid ids form a prefix, are in range, no self loops, no repeats
    assert (np.diff(valid.astype(np.int8), axis=1) <= 0).all()
    assert (adj[valid] < n).all()
    for i in range(n):
        row = adj[i][valid[i]]
        assert len(set(row.tolist())) == row.size and i not in row
    # every node is reachable from the entry point
    seen = np.zeros(n, bool)
    seen[graph._reach_from(np.where(valid, adj.astype(np.int64), -1), ep)] = True
    assert seen.all()
    gt, _ = oracle_lib.bruteforce(w.base, w.queries, 10, w.metric)
    ids, *_ = oracle_lib.search(w.base, adj, ep, w.metric, w.queries, 10, 64)
    rec = np.mean([len(set(ids[i]) & set(gt[i])) / 10 for i in range(len(ids))])
    assert rec >= 0.95, rec


def test_mrng_rule_on_a_line():
    """Points on a line: from the left end, every farther point is shadowed
    by the nearest one (d(1, c) < d(0, c)), so MRNG keeps only one edge."""
    from scattersearch_b200 import graph
    X = torch.tensor([[0.0], [1.0], [2.0], [3.0]])
    cand = torch.tensor([[1, 2, 3]])
    cd = torch.tensor([[1.0, 4.0, 9.0]])
    out = graph.mrng_prune(X, cand, cd, R=3)
    assert out[0].tolist() == [1, -1, -1]


def test_bruteforce_matches_oracle(oracle_lib):
    from scattersearch_b200 import graph
    fx = load_fixture("search_ip_d96")
    X = torch.as_tensor(fx["base"])
    Q = torch.as_tensor(fx["queries"])
    ids, d = graph.bruteforce(X, Q, 10, 1)
    o_ids, _ = oracle_lib.bruteforce(fx["base"], fx["queries"], 10, 1)
    assert (ids.numpy() == o_ids).mean() > 0.99


def test_shard_range_tiles():
    from scattersearch_b200.replicas import shard_range
    for n in (0, 1, 7, 10, 1001):
        for world in (1, 2, 3, 8):
            spans = [shard_range(n, r, world) for r in range(world)]
            assert spans[0][0] == 0 and spans[-1][1] == n
            assert all(spans[i][1] == spans[i + 1][0] for i in range(world - 1))
            sizes = [e - s for s, e in spans]
            assert max(sizes) - min(sizes) <= 1


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _replica_worker(rank, world, port, out_dir):
    import torch.distributed as dist

    from oracle import oracle as O
    from scattersearch_b200.replicas import gather_rows, max_over_ranks, shard_range
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    fx = load_fixture("search_l2_d64")
    s, e = shard_range(len(fx["queries"]), rank, world)
    # each rank searches its own shard of queries on its replica (the oracle
    # stands in for the per-GPU search on CPU)
    ids, _, _, _ = O.search(fx["base"], fx["adj"], int(fx["ep"]), 0, fx["queries"][s:e], 10, 50,
                            nthreads=1)
    allids = gather_rows(ids, len(fx["queries"]), rank, world)
    t = max_over_ranks(float(rank + 1))
    if rank == 0:
        np.save(os.path.join(out_dir, "ids.npy"), allids)
        np.save(os.path.join(out_dir, "t.npy"), np.array([t]))
    dist.destroy_process_group()


def test_replica_sharding_over_gloo(tmp_path, oracle_lib):
    import torch.multiprocessing as mp
    port = _free_port()
    mp.start_processes(_replica_worker, args=(2, port, str(tmp_path)), nprocs=2, join=True,
                       start_method="spawn")
    fx = load_fixture("search_l2_d64")
    one, *_ = oracle_lib.search(fx["base"], fx["adj"], int(fx["ep"]), 0, fx["queries"], 10, 50)
    assert np.array_equal(np.load(tmp_path / "ids.npy"), one)
    assert float(np.load(tmp_path / "t.npy")[0]) == 2.0


def test_autotune_keys_and_cache(tmp_path):
    from scattersearch_b200 import autotune as at
    assert [at.l_bucket(x) for x in (1, 64, 65, 400)] == [1, 64, 128, 512]
    hc = at.hash_candidates(400)
    assert hc[0] == 1024 and hc[-1] == 16384 and all(b == 2 * a for a, b in zip(hc, hc[1:]))
    assert at.hash_candidates(16) == [1024]
    k1 = at.tuning_key("NVIDIA B200", 200, 32, 400)
    assert k1 == at.tuning_key("NVIDIA B200", 200, 32, 300)  # same L bucket
    assert k1 != at.tuning_key("NVIDIA B200", 200, 32, 600)
    path = str(tmp_path / "t" / "tuning.json")
    assert at.load_cache(path) == {}
    at.save_choice(k1, {"warps_per_block": 2, "hash_cap": 2048}, path)
    at.save_choice("other", {"warps_per_block": 1, "hash_cap": 1024}, path)
    data = at.load_cache(path)
    assert data[k1]["hash_cap"] == 2048 and set(data) == {k1, "other"}


def test_autotune_apply_restores_the_whole_layout(tmp_path, monkeypatch):
    """A cached choice sets teams per CTA, table size, stage rows, shared
    stages and the visited-marks mode on the index (a stand-in that records
    the calls; no GPU)."""
    from scattersearch_b200 import autotune as at
    monkeypatch.setattr(at, "_gpu_name", lambda device=None: "GPU-X")

    class FakeIndex:
        dimension, rstride = 96, 32
        calls = []
        marks = []

        def set_tuning(self, *args):
            self.calls.append(args)

        def set_visited_marks(self, mode):
            self.marks.append(mode)

    path = str(tmp_path / "tuning.json")
    idx = FakeIndex()
    assert at.apply(idx, 300, path=path) is None and idx.calls == []
    at.save_choice(at.tuning_key("GPU-X", 96, 32, 300),
                   {"warps_per_block": 4, "hash_cap": 2048, "shared_stages": 3,
                    "stage_rows": 12, "visited_marks": 1}, path)
    assert at.apply(idx, 400, path=path)["hash_cap"] == 2048  # same L bucket (512)
    assert idx.calls == [(4, 2048, 0, 3, 12)] and idx.marks == [1]
    # choices cached before stage layouts existed still apply
    at.save_choice(at.tuning_key("GPU-X", 96, 32, 40), {"warps_per_block": 1, "hash_cap": 1024},
                   path)
    at.apply(idx, 40, path=path)
    assert idx.calls[-1] == (1, 1024, 0, 0, 0) and idx.marks[-1] == 0
    assert len(at.SHARED_CANDIDATES) and all(s < w for w, s in at.SHARED_CANDIDATES)


def test_uneven_recall_helper():
    """Config 4's recall: recall@10 over queries with K >= 10 (their first ten
    ids) and recall@1 over queries with K = 1."""
    import bench
    Ks = np.array([1, 10, 100, 1], np.int32)
    off = np.concatenate([[0], np.cumsum(Ks)[:-1]])
    gt = np.array([np.arange(10) + 100 * i for i in range(4)])
    ids = np.zeros(int(Ks.sum()), np.uint32)
    ids[off[0]] = 0                                # K=1, hit
    ids[off[1]:off[1] + 10] = np.arange(100, 110)  # K=10, all ten
    ids[off[2]:off[2] + 10] = np.r_[200:205, 900:905]  # K=100, five of ten in its first ten
    ids[off[3]] = 999                              # K=1, miss
    r10, r1, n10, n1 = bench.recall_uneven(ids, off, Ks, gt)
    assert (n10, n1) == (2, 2) and r10 == 0.75 and r1 == 0.5


def test_data_tools_split_and_convert(tmp_path):
    """split_fbin keeps the last vectors as queries (scripts/splitfbin.py);
    ann_benchmarks_to_fbin writes base/query/ground truth that the readers
    (and the C ABI loaders' formats) take back unchanged."""
    from scattersearch_b200 import io as sio
    rng = np.random.default_rng(2)
    X = rng.standard_normal((1037, 24)).astype(np.float32)
    src = str(tmp_path / "all.fbin")
    sio.write_fbin(src, X)
    nb, nq, d = sio.split_fbin(src, 37, str(tmp_path / "b.fbin"), str(tmp_path / "q.fbin"))
    assert (nb, nq, d) == (1000, 37, 24)
    assert np.array_equal(sio.load_fbin(str(tmp_path / "b.fbin")), X[:1000])
    assert np.array_equal(sio.load_fbin(str(tmp_path / "q.fbin")), X[1000:])
    with pytest.raises(ValueError):
        sio.split_fbin(src, 2000, str(tmp_path / "x.fbin"), str(tmp_path / "y.fbin"))
    # command line form
    assert sio.main(["split-fbin", src, "--num-queries", "10", "--base-out",
                     str(tmp_path / "b2.fbin"), "--query-out", str(tmp_path / "q2.fbin")]) == 0
    assert sio.load_fbin(str(tmp_path / "q2.fbin")).shape == (10, 24)
    train = rng.standard_normal((500, 16))          # float64, as some HDF5 sets store
    test = rng.standard_normal((20, 16))
    nbr = rng.integers(0, 500, size=(20, 100))
    paths = [str(tmp_path / n) for n in ("base.fbin", "query.fbin", "gt.bin")]
    sio.ann_benchmarks_to_fbin(train, test, nbr, *paths, k=10)
    assert np.array_equal(sio.load_fbin(paths[0]), train.astype(np.float32))
    assert np.array_equal(sio.load_fbin(paths[1]), test.astype(np.float32))
    assert np.array_equal(sio.load_groundtruth(paths[2]), nbr[:, :10].astype(np.uint32))
    with pytest.raises(ValueError):
        sio.ann_benchmarks_to_fbin(train, test, nbr + 500, *paths)


def test_bench_clock_samples_and_profiled_traffic(tmp_path, monkeypatch):
    """The bench's clock record (median SM clock, throttle reasons, the
    one-shot fallback when no sample landed in the window) and the DRAM
    traffic it reads from the committed ncu summary."""
    import bench

    class Done:
        def terminate(self):
            pass

        def wait(self, timeout=None):
            return 0

    rows = ["0, 1965, 1965, 700.1, 0x0, Not Active, Not Active, Not Active, Not Active",
            "0, 1950, 1965, 980.0, 0x4, Not Active, Not Active, Not Active, Active",
            "0, 1965, 1965, 990.5, 0x4, Not Active, Not Active, Not Active, Active"]
    s = bench.ClockSampler(0)
    s.path = str(tmp_path / "clk.csv")
    s.proc = Done()
    s.skip = 1  # a sample from before the warm-up is dropped
    with open(s.path, "w") as f:
        f.write("0, 900, 1965, 100.0, 0x0, Not Active, Active, Not Active, Not Active\n")
        f.write("\n".join(rows) + "\n")
    c = s.stop()
    assert c["samples"] == 3 and c["sm_mhz"] == 1965.0 and c["sm_max_mhz"] == 1965.0
    assert c["reasons"] == ["sw_power_cap"] and c["window"] == "warm-up and timed steps"
    # nothing inside the steps: one read right after them
    s2 = bench.ClockSampler(0)
    s2.path = str(tmp_path / "clk2.csv")
    s2.proc = Done()
    open(s2.path, "w").close()
    monkeypatch.setattr(bench.ClockSampler, "_one_shot", lambda self: rows[:1])
    c2 = s2.stop()
    assert c2["samples"] == 1 and c2["window"] == "right after the timed steps"
    # the roofline's traffic: the committed small-case bytes per evaluated row,
    # scaled by the rows a launch evaluates (10k queries x 6,875 rows here)
    traffic, src = bench.profiled_traffic("cfg3", 10000 * 6875)
    assert ".md:" in src and 5e10 < traffic < 8e10
    assert bench.profiled_traffic("cfg2", 10000 * 6875) == (None, None)
