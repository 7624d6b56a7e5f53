#!/usr/bin/env python
"""Benchmark of the graph-search hot path on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload cfg3|cfg2|cfg1|cfg4] [--L auto|<int>] [--nq Q] [--scale S]

Workload (default): the 1.2M x 200 angular configuration -- seeded
50-component Gaussian mixture, unit-normalised, inner product, K = 100, an
NSG-style graph with out-degree <= 32 built on the device, 10k queries per
GPU.  The beam width L is the smallest of the configuration's values (200,
400, then 800) whose recall@10 against exact brute force is >= 0.95.

One step = one batched persistent search over the whole query batch, with
base, graph and queries resident in HBM (`value`, timed with CUDA events on
the launching stream; the 960 MB base is larger than L2).  `e2e` times the
public C ABI call with pinned host buffers (query upload and result download
inside the timed region).  The plain per-query GPU path (one launch per
query) is timed on a sample beside it.  `cpu_baseline` is the reference's
own SearchArraySimulation (compiled from its sources, -Ofast) on the host
cores over a bounded sample.

--impl reference times that reference CPU search alone as the reference arm
(same workload; rank 0 only under torchrun).

--workload cfg4: one batch of 100k queries with per-query K in {1, 10, 100}
and L in [32, 512] over 5M x 96 unit vectors, searched by one persistent
launch captured in a CUDA graph; its CPU baseline is the oracle's C
restatement (the reference's drivers take one K and L per run).

Multi-GPU (torchrun, one rank per GPU): every rank holds a replica of the
index and searches its own 10k queries (weak scaling, no device collective);
time is the maximum over ranks.
"""
from __future__ import annotations

import argparse
import contextlib
import datetime
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "QPS at recall@10≥0.95, batched vs plain GPU search; p50/p99 online latency"
FALLBACK_HBM_GBS = 6650.0


def log(*a):
    print("[bench]", *a, file=sys.stderr, flush=True)


@contextlib.contextmanager
def stdout_to_stderr():
    """Sends file descriptor 1 to stderr for the duration (the reference
    library prints to stdout; the bench's stdout carries one JSON line)."""
    import ctypes
    sys.stdout.flush()
    libc = ctypes.CDLL(None)
    libc.fflush(None)
    saved = os.dup(1)
    os.dup2(2, 1)
    try:
        yield
    finally:
        libc.fflush(None)
        sys.stdout.flush()
        os.dup2(saved, 1)
        os.close(saved)


def parse_args(argv=None):
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawTextHelpFormatter)
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", default="cfg3", choices=["cfg1", "cfg2", "cfg3", "cfg4"])
    ap.add_argument("--L", default="auto")
    ap.add_argument("--nq", type=int, default=None,
                    help="queries per GPU (default 10000; 100000 for cfg4)")
    ap.add_argument("--scale", type=float, default=1.0, help="base size fraction (profiling)")
    ap.add_argument("--plain-sample", type=int, default=300)
    ap.add_argument("--cpu-seconds", type=float, default=15.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-online", action="store_true",
                    help="skip the serving and intra-query latency legs")
    args = ap.parse_args(argv)
    if args.nq is None:
        args.nq = 100_000 if args.workload == "cfg4" else 10_000
    return args


# --------------------------------------------------------------- plumbing
class Dist:
    def __init__(self, backend):
        self.rank = int(os.environ.get("RANK", "0"))
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.local_rank = int(os.environ.get("LOCAL_RANK", "0"))
        self.pg = False
        if self.world > 1:
            import torch.distributed as dist
            dist.init_process_group(backend, timeout=datetime.timedelta(seconds=600))
            self.pg = True

    def barrier(self):
        if self.pg:
            import torch.distributed as dist
            dist.barrier()

    def max(self, v, device=None):
        from scattersearch_b200.replicas import max_over_ranks
        return max_over_ranks(v, device) if self.pg else float(v)

    def close(self):
        if self.pg:
            import torch.distributed as dist
            dist.destroy_process_group()


class ClockSampler:
    """nvidia-smi samples every 50 ms while the GPU runs the warm-up and timed
    steps (a timed region of a few 16 ms steps is shorter than nvidia-smi's
    usual interval, so sampling starts before the warm-up, and the samples
    taken before it are dropped)."""
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.path = None
        self.skip = 0

    def _lines(self):
        try:
            with open(self.path) as f:
                return f.read().splitlines()
        except OSError:
            return []

    def start(self):
        """Starts sampling and returns once the first sample is written (at
        most 3 s), so that the steps that follow are covered."""
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "50"],
                stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None
            return
        t0 = time.time()
        while time.time() - t0 < 3.0 and not self._lines():
            time.sleep(0.01)
        self.skip = len(self._lines())

    def _one_shot(self):
        try:
            out = subprocess.run(["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.FIELDS}",
                                  "--format=csv,noheader,nounits"], capture_output=True,
                                 text=True, timeout=10).stdout
            return out.splitlines()
        except (OSError, subprocess.SubprocessError):
            return []

    def stop(self):
        if self.proc is None:
            return None
        time.sleep(0.06)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        lines = self._lines()[self.skip:]
        os.unlink(self.path)
        window = "warm-up and timed steps"
        if not lines:  # no sample landed inside the steps: read once right after them
            lines, window = self._one_shot(), "right after the timed steps"
        rows = [[p.strip() for p in line.split(",")] for line in lines]
        rows = [r for r in rows if len(r) >= 9]
        if not rows:
            return None
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if "Active" in r[5 + i]
                          and "Not" not in r[5 + i]})
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": reasons,
                "samples": len(rows), "window": window}


PROFILED_TRAFFIC = {
    # (workload, L, queries) -> ncu summary holding the DRAM bytes of one launch
    ("cfg3", 400, 10000): "profiles/warp_search_kernel_1.2Mx200_ip_L400.md",
}


def profiled_traffic(workload, L, nq):
    """DRAM bytes (read + write) of one search launch from the committed ncu
    summary of this exact workload, or None when none was captured."""
    rel = PROFILED_TRAFFIC.get((workload, L, nq))
    if not rel:
        return None, None
    try:
        with open(os.path.join(ROOT, rel)) as f:
            for line in f:
                if line.startswith("traffic_bytes_per_launch:"):
                    return float(line.split(":", 1)[1]), rel
    except OSError:
        pass
    return None, None


def measured_hbm_peak():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return FALLBACK_HBM_GBS, "fallback"


# --------------------------------------------------------------- workload
def workload_spec(name):
    if name == "cfg4":
        return dict(cfg=4, Ls=[], K=100, desc="5Mx96 angular (IP), per-query K in {1,10,100} "
                                               "and L in [32,512]", gt_sample=10000)
    if name == "cfg3":
        return dict(cfg=3, Ls=[200, 400, 800], K=100, desc="1.2Mx200 angular (IP), K=100")
    if name == "cfg2":
        return dict(cfg=2, Ls=[64, 128, 256], K=10, desc="1Mx128 uint8-valued, L2, K=10")
    return dict(cfg=1, Ls=[100, 200], K=10, desc="100kx200 L2, K=10")


def build_workload(args, rank, world, device):
    """Seeded data, NSG-style graph and exact ground truth (setup, untimed)."""
    import torch
    from scattersearch_b200 import datasets, graph
    spec = workload_spec(args.workload)
    t0 = time.time()
    w = datasets.config(spec["cfg"], scale=args.scale, n_queries=args.nq * world)
    queries = np.ascontiguousarray(w.queries[rank * args.nq:(rank + 1) * args.nq])
    log(f"data {w.base.shape} queries {queries.shape} in {time.time() - t0:.1f}s")
    t0 = time.time()
    X = torch.from_numpy(w.base).to(device)
    # config 4 takes its exact 64-NN from the library's tensor-core brute force
    backend = "bruteforce" if spec["cfg"] == 4 and device != "cpu" else "torch"
    adj, ep = graph.build_graph(X, R=w.graph_R, knn_k=w.graph_knn, device=device,
                                knn_backend=backend)
    log(f"graph R={w.graph_R} ep={ep} mean degree {(adj != 0xFFFFFFFF).sum(1).mean():.1f} "
        f"in {time.time() - t0:.1f}s")
    Q = torch.from_numpy(queries).to(device)
    if device != "cpu" and torch.cuda.is_available():
        torch.cuda.empty_cache()  # hand the graph build's scratch back to the driver
    ns = min(len(queries), spec.get("gt_sample", len(queries)))
    gt, gt_info = ground_truth(X, Q[:ns], w.metric, device)
    log(f"ground truth: {gt_info}")
    return dict(spec=spec, w=w, X=X, queries=queries, Q=Q, adj=adj, ep=ep,
                gt=gt, gt_info=gt_info, metric=w.metric, K=spec["K"])


def ground_truth(X, Q, metric, device, k=10):
    """Exact top-10 of every query: the library's tensor-core brute force
    (timed with CUDA events), or torch when the library is not built."""
    import torch
    nq, dim = Q.shape
    n = X.shape[0]
    try:
        from scattersearch_b200 import ANNSearch
        idx = ANNSearch(dim, n, X, metric, base_on_device=True)
    except Exception as e:  # library missing (e.g. a CPU-only run)
        from scattersearch_b200 import graph
        gt, _ = graph.bruteforce(X, Q, k, metric)
        return gt.cpu().numpy(), {"kernel": f"torch ({e.__class__.__name__})"}
    ids = torch.empty((nq, k), dtype=torch.int32, device=device)
    st = torch.cuda.current_stream()
    idx.bruteforce_device(Q, nq, k, ids, stream=st.cuda_stream)  # warm-up (norms, attributes)
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record(st)
    idx.bruteforce_device(Q, nq, k, ids, stream=st.cuda_stream)
    b.record(st)
    torch.cuda.synchronize()
    ms = a.elapsed_time(b)
    idx.close()
    return ids.cpu().numpy().view(np.uint32), {
        "kernel": "bf_tc_candidates_kernel (tcgen05.mma kind::tf32 into TMEM, three-term "
                  "products, FP32 accumulate) + bf_rerank_kernel (exact FP32 distance, ties by id)",
        "ms": ms, "tensor_tflops": 3 * 2 * nq * n * dim / ms / 1e9,
        "queries": int(nq), "base": int(n)}


def recall_at_10(ids, gt):
    ids = np.asarray(ids)[:, :10].astype(np.int64)
    hit = [(np.isin(ids[i], gt[i])).sum() for i in range(len(ids))]
    return float(np.mean(hit) / 10.0)


# -------------------------------------------------------- reference arm
def cpu_threads():
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


def time_reference(wl, L, seconds, fast=True, warm=1):
    with stdout_to_stderr():
        return _time_reference(wl, L, seconds, fast, warm)


def _time_reference(wl, L, seconds, fast=True, warm=1):
    """Reference SearchArraySimulation on the host cores over a bounded
    sample; returns (qps, sample size, ids of the sample, threads)."""
    from oracle import oracle as O
    th = cpu_threads()
    ref = O.RefIndex(wl["w"].base, wl["metric"], wl["adj"], wl["ep"], fast=fast)
    K = wl["K"]
    q = wl["queries"]
    probe = min(len(q), max(8 * th, 32))
    t0 = time.perf_counter()
    ref.search(q[:probe], K, L, nthreads=th)
    rate = probe / max(1e-6, time.perf_counter() - t0)
    sample = int(min(len(q), max(probe, rate * seconds)))
    reps = max(1, int(round(rate * seconds / sample)))
    for _ in range(warm):
        ref.search(q[:min(sample, probe)], K, L, nthreads=th)
    t0 = time.perf_counter()
    for _ in range(reps):
        ids = ref.search(q[:sample], K, L, nthreads=th)
    dt = time.perf_counter() - t0
    ref.close()
    return sample * reps / dt, (sample, reps), ids, th


def run_reference_arm(args):
    with stdout_to_stderr():
        out = _reference_arm(args)
    if out is not None:
        print(json.dumps(out))
    return 0


def _reference_arm(args):
    d = Dist("gloo")
    if d.rank != 0:
        d.close()
        return None
    import torch
    from oracle import oracle as O
    if args.workload == "cfg4":
        d.close()
        return {"impl": "reference", "unavailable": "the reference's drivers take one K and L "
                "per run; per-query K/L batches have no reference entry point"}
    if not O.have_reference(fast=True):
        d.close()
        return {"impl": "reference", "unavailable": "oracle/_ref/libssref_fast.so was not built"}
    device = torch.device("cuda", d.local_rank) if torch.cuda.is_available() else "cpu"
    wl = build_workload(args, 0, 1, device)
    L = choose_L_reference(args, wl)
    th = cpu_threads()
    ref = O.RefIndex(wl["w"].base, wl["metric"], wl["adj"], wl["ep"], fast=True)
    K, q = wl["K"], wl["queries"]
    probe = min(len(q), max(8 * th, 32))
    t0 = time.perf_counter()
    ref.search(q[:probe], K, L, nthreads=th)
    rate = probe / max(1e-6, time.perf_counter() - t0)
    # a step is a bounded sample of the workload: about cpu_seconds/steps of
    # host work, the whole batch repeated when it is shorter than that
    per_step = int(min(len(q), max(probe, rate * args.cpu_seconds / max(1, args.steps))))
    reps = max(1, int(round(rate * args.cpu_seconds / max(1, args.steps) / per_step)))
    for _ in range(args.warmup):
        ref.search(q[:min(per_step, probe)], K, L, nthreads=th)
    times = []
    ids = None
    for s in range(args.steps):
        t0 = time.perf_counter()
        for _ in range(reps):
            ids = ref.search(q[:per_step], K, L, nthreads=th)
        times.append(time.perf_counter() - t0)
    ref.close()
    total = sum(times)
    qps = per_step * reps * args.steps / total
    rec = recall_at_10(ids, wl["gt"][:per_step])
    sample = (f"first {per_step} of {len(q)} queries x{reps} per step, K={K}, L={L}, "
              f"-Ofast build, OpenMP over queries, one visited bitset per thread")
    out = {
        "impl": "reference", "metric": METRIC, "value": qps, "unit": "queries/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1000 * total / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": wl["w"].name + " (synthetic, seeded)",
        "config": {"workload": wl["spec"]["desc"], "K": K, "L": L, "nq_per_step": per_step,
                   "recall@10": rec, "graph": "NSG-style, R<=32, built on the device (setup)"},
        "cpu_baseline": {"value": qps, "unit": "queries/s", "cores": th, "kind": "reference",
                         "sample": sample},
        "e2e": {"value": qps, "unit": "queries/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    d.close()
    return out


def choose_L_reference(args, wl):
    if args.L != "auto":
        return int(args.L)
    # same rule as our arm: smallest configured L whose GPU-free recall check
    # passes is not affordable on the host, so use the GPU search to pick it
    # when the library is present, else the largest configured L.
    try:
        from scattersearch_b200 import ANNSearch
        idx = ANNSearch(wl["X"].shape[1], wl["X"].shape[0], wl["X"], wl["metric"],
                        base_on_device=True)
        idx.SetGraph(wl["adj"], wl["ep"])
        L = pick_L(idx, wl)[0]
        idx.close()
        return L
    except Exception as e:  # library missing: fall back to the configured maximum
        log(f"L selection without the GPU library ({e}); using the largest configured L")
        return wl["spec"]["Ls"][-1]


# -------------------------------------------------------------- our arm
def pick_L(idx, wl, target=0.95):
    res = []
    for L in wl["spec"]["Ls"]:
        ids, _ = idx.search_batch(wl["queries"], wl["K"], L)
        r = recall_at_10(ids, wl["gt"])
        res.append((L, r))
        log(f"L={L} recall@10={r:.4f}")
        if r >= target:
            return L, r, res
    return res[-1][0], res[-1][1], res


def measure_online(idx, wl, L, rates=(100_000, 300_000, 550_000), seconds=0.15):
    """Serving leg: Poisson arrivals replayed through the continuous-batching
    server (ss_server_replay); latency is arrival to result on the host."""
    from scattersearch_b200.serving import Server, poisson_arrivals
    K = wl["K"]
    Q = wl["queries"]
    out = []
    with Server(idx, max_batch=512, max_inflight=4, K_max=K, L_max=L) as srv:
        warm = min(len(Q), 4096)
        srv.replay(Q[:warm], np.full(warm, K, np.int32), np.full(warm, L, np.int32),
                   poisson_arrivals(warm, 100_000, seed=1))
        srv.stats(reset=True)
        for rate in rates:
            n = int(max(2000, rate * seconds))
            q = Q[np.arange(n) % len(Q)]
            t0 = time.perf_counter()
            _, _, _, lat = srv.replay(q, np.full(n, K, np.int32), np.full(n, L, np.int32),
                                      poisson_arrivals(n, rate, seed=rate))
            wall = time.perf_counter() - t0
            st = srv.stats(reset=True)
            out.append({"offered_qps": rate, "requests": n, "sustained_qps": n / wall,
                        "p50_ms": float(np.percentile(lat, 50)) / 1e3,
                        "p99_ms": float(np.percentile(lat, 99)) / 1e3,
                        "p999_ms": float(np.percentile(lat, 99.9)) / 1e3,
                        "mean_batch": st["mean_batch"]})
            log(f"online {rate}/s: p50 {out[-1]['p50_ms']:.2f} ms p99 {out[-1]['p99_ms']:.2f} ms")
    return {"K": K, "L": L, "max_batch": 512, "slots": 4, "arrivals": "Poisson",
            "latency": "arrival to result on the host", "rates": out}


def measure_intra_latency(idx, wl, L, device, batches=(1, 4, 16), widths=(4, 8, 16), reps=10):
    """Device time of one small batch: the plain kernel (one warp per query)
    and the intra-query kernel (one CTA of W warps per query, W candidates
    expanded per step), with recall@10 of each."""
    import torch
    K = wl["K"]
    Q = wl["Q"]
    st = torch.cuda.current_stream()
    res = []
    idx.set_tuning()  # the tuned table size is the batched kernel's; use automatic sizes here
    for b in batches:
        ids = torch.empty((b, K), dtype=torch.int32, device=device)
        row = {"batch": b}
        for W in (0,) + tuple(widths):
            ms, hits = [], []
            for r in range(reps):
                q = Q[r * b:(r + 1) * b]
                run = (lambda: idx.search_batch_device(q, b, ids, None, K=K, L=L,
                                                       stream=st.cuda_stream)) if W == 0 else \
                      (lambda: idx.search_intra_batch_device(q, b, K, L, W, ids,
                                                             stream=st.cuda_stream))
                run()
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record(st)
                run()
                e1.record(st)
                torch.cuda.synchronize()
                ms.append(e0.elapsed_time(e1))
                hits.append(recall_at_10(ids.cpu().numpy().view(np.uint32),
                                         wl["gt"][r * b:(r + 1) * b]))
            key = "plain" if W == 0 else f"intra_w{W}"
            row[key] = {"ms": float(np.median(ms)), "recall@10": float(np.mean(hits))}
        for W in (w for w in widths if w <= 8):  # ScatterSearch's form: a pool per warp, ET
            ms, hits = [], []
            for r in range(reps):
                q = Q[r * b:(r + 1) * b]
                run = lambda: idx.search_scatter_device(q, b, K, L, W, ids, early_termination=True,
                                                        seed=r + 1, stream=st.cuda_stream)
                run()
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record(st)
                run()
                e1.record(st)
                torch.cuda.synchronize()
                ms.append(e0.elapsed_time(e1))
                hits.append(recall_at_10(ids.cpu().numpy().view(np.uint32),
                                         wl["gt"][r * b:(r + 1) * b]))
            row[f"scatter_et_w{W}"] = {"ms": float(np.median(ms)), "recall@10": float(np.mean(hits))}
        res.append(row)
        log(f"batch {b}: " + ", ".join(f"{k} {v['ms']:.2f} ms" for k, v in row.items()
                                          if k != "batch"))
    return {"K": K, "L": L, "timing": "CUDA events, median of %d batches" % reps, "rows": res}


def run_ours(args):
    import torch
    d = Dist("nccl")
    torch.cuda.set_device(d.local_rank)
    device = torch.device("cuda", d.local_rank)
    from scattersearch_b200 import ANNSearch
    wl = build_workload(args, d.rank, d.world, device)
    K = wl["K"]
    nq, dim = wl["queries"].shape
    idx = ANNSearch(dim, wl["X"].shape[0], wl["X"], wl["metric"], base_on_device=True)
    idx.SetGraph(wl["adj"], wl["ep"])

    if args.L == "auto":
        L, rec, sweep = pick_L(idx, wl)
    else:
        L = int(args.L)
        ids, _ = idx.search_batch(wl["queries"], K, L)
        rec, sweep = recall_at_10(ids, wl["gt"]), []
    # every rank must use the same L
    if d.pg:
        import torch.distributed as dist
        t = torch.tensor([L], device=device)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        L = int(t.item())

    # launch layout (teams per CTA, visited-table size) tuned on a sample
    from scattersearch_b200 import autotune
    tune = autotune.autotune(idx, wl["Q"], K, L, reps=2, path=None)
    for r in sorted(tune["table"], key=lambda r: r["ms"])[:6]:
        log(f"  layout {r}")
    log(f"tuned: {tune['warps_per_block']} teams per CTA, {tune['shared_stages']} shared stages "
        f"(0 = one per team) of {tune['stage_rows']} rows, {tune['hash_cap']}-slot visited table")

    Qd = wl["Q"]
    ids_d = torch.empty((nq, K), dtype=torch.int32, device=device)
    dist_d = torch.empty((nq, K), dtype=torch.float32, device=device)
    ndc_d = torch.empty(nq, dtype=torch.int32, device=device)
    hops_d = torch.empty(nq, dtype=torch.int32, device=device)
    stream = torch.cuda.current_stream()

    def step(with_stats=False):
        if with_stats:
            idx.search_batch_device(Qd, nq, ids_d, dist_d, K=K, L=L, ndc=ndc_d, hops=hops_d,
                                    stream=stream.cuda_stream)
        else:  # the launch captured in a CUDA graph, replayed
            plan.launch(stream.cuda_stream)

    # Stats passes (same traversal, same ids).  The algorithmic bytes count
    # the reference algorithm's distance evaluations, taken with a visited
    # table large enough never to forget; the default table may forget ids
    # and evaluate them again, which the second pass counts.
    idx.set_tuning(hash_cap=65536)
    step(with_stats=True)
    torch.cuda.synchronize()
    if idx.batch_status():
        raise RuntimeError("device batch reported failed queries")
    ndc = ndc_d.cpu().numpy().astype(np.int64)
    hops = hops_d.cpu().numpy().astype(np.int64)
    ids_exact = ids_d.cpu().numpy().copy()
    idx.set_tuning(tune["warps_per_block"], tune["hash_cap"], 0, tune["shared_stages"],
                   tune["stage_rows"])
    step(with_stats=True)
    torch.cuda.synchronize()
    ndc_dev = ndc_d.cpu().numpy().astype(np.int64)
    if not np.array_equal(ids_d.cpu().numpy(), ids_exact):
        raise RuntimeError("ids depend on the visited-table size")
    plan = idx.plan_batch_device(Qd, nq, K, L, ids_d, dist_d)
    rstride = idx.rstride
    bytes_per_step = float(ndc.sum() * 4 * dim + hops.sum() * 4 * rstride + nq * 4 * dim)
    row_bytes = 4 * ((dim + 7) // 8 * 8)
    device_bytes_per_step = float(ndc_dev.sum() * row_bytes + hops.sum() * 4 * rstride
                                  + nq * 4 * dim)

    sampler = ClockSampler(d.local_rank)
    sampler.start()
    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    d.barrier()
    torch.cuda.nvtx.range_push("timed")
    evs = []
    for _ in range(args.steps):
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record(stream)
        step()
        e.record(stream)
        evs.append((s, e))
    torch.cuda.synchronize()
    torch.cuda.nvtx.range_pop()
    d.barrier()
    clocks = sampler.stop()
    step_ms = [s.elapsed_time(e) for s, e in evs]
    if plan.failed_queries():
        raise RuntimeError("graph-captured search reported failed queries")
    total_s = d.max(sum(step_ms) / 1000.0, device)
    qps = nq * d.world * args.steps / total_s
    ids_np = ids_d.cpu().numpy().view(np.uint32)
    rec_timed = recall_at_10(ids_np, wl["gt"])

    # e2e: public C ABI with pinned host buffers
    qh = torch.empty((nq, dim), dtype=torch.float32).pin_memory()
    qh.numpy()[:] = wl["queries"]
    ih = torch.empty((nq, K), dtype=torch.int32).pin_memory()
    dh = torch.empty((nq, K), dtype=torch.float32).pin_memory()
    qn, idn, dn = qh.numpy(), ih.numpy().view(np.uint32), dh.numpy()
    for _ in range(max(1, args.warmup)):
        idx.search_batch(qn, K, L, out_ids=idn, out_dists=dn)
    d.barrier()
    torch.cuda.synchronize()
    e2e_t = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        idx.search_batch(qn, K, L, out_ids=idn, out_dists=dn)
        e2e_t.append(time.perf_counter() - t0)
    e2e_s = d.max(sum(e2e_t), device)
    e2e_qps = nq * d.world * args.steps / e2e_s
    same_ids = bool(np.array_equal(idn, ids_np))

    # plain per-query GPU path on a sample
    ns = min(args.plain_sample, nq)
    for i in range(min(8, ns)):
        idx.search(wl["queries"][i], K, L)
    t0 = time.perf_counter()
    plain_ids = np.empty((ns, K), dtype=np.uint32)
    for i in range(ns):
        plain_ids[i], _ = idx.search(wl["queries"][i], K, L)
    plain_s = time.perf_counter() - t0
    plain_qps = ns / plain_s
    plain_same = bool(np.array_equal(plain_ids, ids_np[:ns]))

    online = None if args.no_online else measure_online(idx, wl, L)
    intra = None if args.no_online else measure_intra_latency(idx, wl, L, device)
    idx.set_tuning(tune["warps_per_block"], tune["hash_cap"], 0, tune["shared_stages"],
                   tune["stage_rows"])

    peak, peak_kind = measured_hbm_peak()
    traffic, traffic_src = profiled_traffic(args.workload, L, nq)
    mean_step_s = sum(step_ms) / len(step_ms) / 1000.0
    achieved = bytes_per_step / mean_step_s / 1e9

    out = {
        "metric": METRIC, "value": qps, "unit": "queries/s", "n_gpus": d.world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000 * total_s / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": wl["w"].name + " (synthetic, seeded numpy; graph built on the device)",
        "config": {"workload": wl["spec"]["desc"] + f", {nq} queries per GPU, batched persistent",
                   "K": K, "L": L, "recall@10": rec_timed, "L_sweep": sweep,
                   "base": list(wl["X"].shape), "graph_R": int(wl["w"].graph_R),
                   "mean_degree": float((wl["adj"] != 0xFFFFFFFF).sum(1).mean()),
                   "l2": "inputs larger than L2 (base %.0f MB > 126 MB L2)"
                         % (wl["X"].numel() * 4 / 1e6),
                   "parallelism": f"replicas x{d.world}, queries sharded",
                   "ground_truth": wl["gt_info"],
                   "tuning": {"warps_per_block": tune["warps_per_block"],
                              "shared_stages": tune["shared_stages"],
                              "stage_rows": tune["stage_rows"],
                              "hash_cap": tune["hash_cap"],
                              "sample": f"the {nq} bench queries (launch layout only)"}},
        "e2e": {"value": e2e_qps, "unit": "queries/s", "h2d_bytes_per_step": nq * dim * 4,
                "d2h_bytes_per_step": nq * K * 8, "ids_equal_device_path": same_ids},
        "plain_gpu": {"value": plain_qps, "unit": "queries/s", "sample": ns,
                      "ids_equal_batched": plain_same,
                      "batched_over_plain": qps / d.world / plain_qps},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "peak_source": peak_kind, "traffic": traffic,
                     "traffic_source": traffic_src,
                     "algorithmic_bytes_per_query": bytes_per_step / nq,
                     "ndc_per_query": float(ndc.mean()), "hops_per_query": float(hops.mean()),
                     "distance_evals_per_s": float(ndc.sum()) / mean_step_s,
                     "device_evals_per_query": float(ndc_dev.mean()),
                     "device_row_gbps": device_bytes_per_step / mean_step_s / 1e9},
        "online": online,
        "intra_latency": intra,
        "gpu_launches": args.steps,
        "launch": "one CUDA graph per step (queue reset, status reset, search kernel)",
        "clocks": clocks,
    }
    if d.rank == 0 and d.world == 1 and not args.no_cpu_baseline:
        from oracle import oracle as O
        kind = "reference" if O.have_reference(fast=True) else None
        if kind:
            cqps, (sample, reps), cids, th = time_reference(wl, L, args.cpu_seconds)
            out["cpu_baseline"] = {
                "value": cqps, "unit": "queries/s", "cores": th, "kind": kind,
                "sample": f"first {sample} of {nq} queries x{reps} passes, K={K}, L={L}, "
                          "reference SearchArraySimulation built -Ofast, OpenMP over queries, "
                          "one visited bitset per thread",
                "ids_equal_gpu_fraction": float((cids == ids_np[:sample]).all(1).mean())}
        else:
            out["cpu_baseline"] = None
    plan.close()
    idx.close()
    if d.rank == 0:
        print(json.dumps(out))
    d.close()
    return 0

def recall_uneven(ids_flat, off, Ks, gt):
    """recall@10 over the sampled queries with K >= 10 and recall@1 over those
    with K = 1 (query i's list starts at off[i])."""
    r10, r1 = [], []
    for i in range(len(gt)):
        k = int(Ks[i])
        got = ids_flat[off[i]:off[i] + min(k, 10)].astype(np.int64)
        if k >= 10:
            r10.append(np.isin(got, gt[i]).sum() / 10.0)
        else:
            r1.append(float(got[0] == gt[i][0]))
    return (float(np.mean(r10)) if r10 else None, float(np.mean(r1)) if r1 else None,
            len(r10), len(r1))


def run_uneven(args):
    """Config 4: one batch with per-query K and L, searched by one persistent
    launch captured in a CUDA graph (ss_plan_create_uneven)."""
    import torch
    d = Dist("nccl")
    torch.cuda.set_device(d.local_rank)
    device = torch.device("cuda", d.local_rank)
    from scattersearch_b200 import ANNSearch, autotune, datasets
    wl = build_workload(args, d.rank, d.world, device)
    nq, dim = wl["queries"].shape
    Ks, Ls = datasets.uneven_k_l(nq * d.world)
    Ks = np.ascontiguousarray(Ks[d.rank * nq:(d.rank + 1) * nq])
    Ls = np.ascontiguousarray(Ls[d.rank * nq:(d.rank + 1) * nq])
    off = np.concatenate([[0], np.cumsum(Ks.astype(np.int64))[:-1]]).astype(np.int64)
    total = int(Ks.sum())
    L_max = int(Ls.max())
    idx = ANNSearch(dim, wl["X"].shape[0], wl["X"], wl["metric"], base_on_device=True)
    idx.SetGraph(wl["adj"], wl["ep"])
    Qd = wl["Q"]
    dK, dL, doff = (torch.from_numpy(a).to(device) for a in (Ks, Ls, off))
    tune = autotune.autotune(idx, Qd, total, L_max, reps=2, path=None, Ks=dK, Ls=dL,
                             out_off=doff)
    log(f"tuned: {tune['warps_per_block']} teams per CTA, {tune['shared_stages']} shared stages "
        f"(0 = one per team) of {tune['stage_rows']} rows, {tune['hash_cap']}-slot visited table")
    ids_d = torch.empty(total, dtype=torch.int32, device=device)
    dist_d = torch.empty(total, dtype=torch.float32, device=device)
    ndc_d = torch.empty(nq, dtype=torch.int32, device=device)
    hops_d = torch.empty(nq, dtype=torch.int32, device=device)
    stream = torch.cuda.current_stream()

    def stats_pass():
        idx.search_batch_device(Qd, nq, ids_d, dist_d, Ks=dK, Ls=dL, out_off=doff, L_max=L_max,
                                ndc=ndc_d, hops=hops_d, stream=stream.cuda_stream)
        torch.cuda.synchronize()
        if idx.batch_status():
            raise RuntimeError("device batch reported failed queries")

    idx.set_tuning(hash_cap=65536)  # exact distance-evaluation counts
    stats_pass()
    ndc = ndc_d.cpu().numpy().astype(np.int64)
    hops = hops_d.cpu().numpy().astype(np.int64)
    ids_exact = ids_d.cpu().numpy().copy()
    idx.set_tuning(tune["warps_per_block"], tune["hash_cap"], 0, tune["shared_stages"],
                   tune["stage_rows"])
    stats_pass()
    ndc_dev = ndc_d.cpu().numpy().astype(np.int64)
    if not np.array_equal(ids_d.cpu().numpy(), ids_exact):
        raise RuntimeError("ids depend on the visited-table size")
    plan = idx.plan_batch_uneven_device(Qd, nq, dK, dL, doff, L_max, ids_d, dist_d)
    rstride = idx.rstride
    bytes_per_step = float(ndc.sum() * 4 * dim + hops.sum() * 4 * rstride + nq * 4 * dim)

    sampler = ClockSampler(d.local_rank)
    sampler.start()
    for _ in range(args.warmup):
        plan.launch(stream.cuda_stream)
    torch.cuda.synchronize()
    d.barrier()
    evs = []
    for _ in range(args.steps):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        plan.launch(stream.cuda_stream)
        b.record(stream)
        evs.append((a, b))
    torch.cuda.synchronize()
    d.barrier()
    clocks = sampler.stop()
    step_ms = [a.elapsed_time(b) for a, b in evs]
    if plan.failed_queries():
        raise RuntimeError("graph-captured search reported failed queries")
    total_s = d.max(sum(step_ms) / 1000.0, device)
    qps = nq * d.world * args.steps / total_s
    ids_np = ids_d.cpu().numpy().view(np.uint32)
    if not np.array_equal(ids_np, ids_exact.view(np.uint32)):
        raise RuntimeError("graph replay returned other ids than the direct launch")
    r10, r1, n10, n1 = recall_uneven(ids_np, off, Ks, wl["gt"])

    # e2e: public C ABI (ss_search_batch_uneven) with pinned host buffers
    qh = torch.empty((nq, dim), dtype=torch.float32).pin_memory()
    qh.numpy()[:] = wl["queries"]
    ih = torch.empty(total, dtype=torch.int32).pin_memory()
    dh = torch.empty(total, dtype=torch.float32).pin_memory()
    qn, idn, dn = qh.numpy(), ih.numpy().view(np.uint32), dh.numpy()
    for _ in range(max(1, args.warmup)):
        idx.search_batch_uneven(qn, Ks, Ls, out_ids=idn, out_dists=dn)
    d.barrier()
    e2e_t = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        idx.search_batch_uneven(qn, Ks, Ls, out_ids=idn, out_dists=dn)
        e2e_t.append(time.perf_counter() - t0)
    e2e_s = d.max(sum(e2e_t), device)
    e2e_qps = nq * d.world * args.steps / e2e_s
    same_ids = bool(np.array_equal(idn, ids_np))

    # plain per-query GPU path on a sample
    ns = min(args.plain_sample, nq)
    for i in range(min(8, ns)):
        idx.search(wl["queries"][i], int(Ks[i]), int(Ls[i]))
    plain_same = True
    t0 = time.perf_counter()
    for i in range(ns):
        got, _ = idx.search(wl["queries"][i], int(Ks[i]), int(Ls[i]))
        plain_same &= bool(np.array_equal(got, ids_np[off[i]:off[i] + Ks[i]]))
    plain_qps = ns / (time.perf_counter() - t0)

    peak, peak_kind = measured_hbm_peak()
    traffic, traffic_src = profiled_traffic(args.workload, L_max, nq)
    mean_step_s = sum(step_ms) / len(step_ms) / 1000.0
    achieved = bytes_per_step / mean_step_s / 1e9
    out = {
        "metric": METRIC, "value": qps, "unit": "queries/s", "n_gpus": d.world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000 * total_s / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": wl["w"].name + " (synthetic, seeded numpy; graph built on the device)",
        "config": {"workload": wl["spec"]["desc"] + f", {nq} queries per GPU, one "
                   "graph-captured persistent launch",
                   "K_counts": {str(k): int((Ks == k).sum()) for k in (1, 10, 100)},
                   "L_mean": float(Ls.mean()), "L_max": L_max,
                   "recall@10_K>=10": r10, "recall@1_K=1": r1,
                   "recall_sample": f"first {len(wl['gt'])} queries ({n10} with K>=10, "
                                    f"{n1} with K=1)",
                   "base": list(wl["X"].shape), "graph_R": int(wl["w"].graph_R),
                   "mean_degree": float((wl["adj"] != 0xFFFFFFFF).sum(1).mean()),
                   "l2": "inputs larger than L2 (base %.0f MB > 126 MB L2)"
                         % (wl["X"].numel() * 4 / 1e6),
                   "parallelism": f"replicas x{d.world}, queries sharded",
                   "ground_truth": wl["gt_info"],
                   "tuning": {"warps_per_block": tune["warps_per_block"],
                              "shared_stages": tune["shared_stages"],
                              "stage_rows": tune["stage_rows"],
                              "hash_cap": tune["hash_cap"]}},
        "e2e": {"value": e2e_qps, "unit": "queries/s", "h2d_bytes_per_step": nq * dim * 4,
                "d2h_bytes_per_step": total * 8, "ids_equal_device_path": same_ids},
        "plain_gpu": {"value": plain_qps, "unit": "queries/s", "sample": ns,
                      "ids_equal_batched": plain_same,
                      "batched_over_plain": qps / d.world / plain_qps},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "peak_source": peak_kind, "traffic": traffic,
                     "traffic_source": traffic_src,
                     "algorithmic_bytes_per_query": bytes_per_step / nq,
                     "ndc_per_query": float(ndc.mean()), "hops_per_query": float(hops.mean()),
                     "distance_evals_per_s": float(ndc.sum()) / mean_step_s,
                     "device_evals_per_query": float(ndc_dev.mean())},
        "gpu_launches": args.steps,
        "launch": "one CUDA graph per step (queue reset, status reset, search kernel)",
        "clocks": clocks,
    }
    if d.rank == 0 and d.world == 1 and not args.no_cpu_baseline:
        out["cpu_baseline"] = time_port_uneven(wl, Ks, Ls, off, ids_np, args.cpu_seconds)
    plan.close()
    idx.close()
    if d.rank == 0:
        print(json.dumps(out))
    d.close()
    return 0


def time_port_uneven(wl, Ks, Ls, off, ids_np, seconds):
    """The oracle's C restatement of SearchArraySimulation, OpenMP over
    queries with per-query K and L, on a bounded prefix of the batch (the
    reference's own drivers take one K and L per run)."""
    from oracle import oracle as O
    th = cpu_threads()
    base, adj, ep, metric, q = wl["w"].base, wl["adj"], int(wl["ep"]), wl["metric"], wl["queries"]
    probe = min(len(q), max(8 * th, 64))
    t0 = time.perf_counter()
    O.search(base, adj, ep, metric, q[:probe], Ks=Ks[:probe], Ls=Ls[:probe], nthreads=th)
    rate = probe / max(1e-6, time.perf_counter() - t0)
    sample = int(min(len(q), max(probe, rate * seconds)))
    t0 = time.perf_counter()
    cids = O.search(base, adj, ep, metric, q[:sample], Ks=Ks[:sample], Ls=Ls[:sample],
                    nthreads=th)[0]
    dt = time.perf_counter() - t0
    n_ids = int(off[sample - 1] + Ks[sample - 1]) if sample else 0
    return {"value": sample / dt, "unit": "queries/s", "cores": th, "kind": "port",
            "sample": f"first {sample} of {len(q)} queries, per-query K and L, C restatement "
                      "of SearchArraySimulation, OpenMP over queries",
            "ids_equal_gpu": bool(np.array_equal(cids, ids_np[:n_ids]))}


def main(argv=None):
    args = parse_args(argv)
    if args.impl == "reference":
        return run_reference_arm(args)
    if args.workload == "cfg4":
        return run_uneven(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
