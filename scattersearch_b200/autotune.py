"""Launch autotuner of the batched search kernel.

The reference has no tunables beyond compile-time macros.  Here the batched
warp-per-query kernel exposes three layout choices that change speed but never
results: how many query teams share a CTA (``warps_per_block``), how many row
stages those teams share (``shared_stages``; 0 = one per team, fewer stages
than teams leave room for more teams per SM) and the size of each query's
shared-memory visited table (``hash_cap``; a smaller table fits more teams
per SM but forgets more visited ids, which are then evaluated again).  A
fourth choice, the visited marks in device memory behind that table
(``visited_marks``), stops those repeats at the cost of a mark read where a
bucket has evicted: at 1.2M x 200 they are worth 5% at L = 400 and cost 12%
at L = 200, so they are timed too.  ``autotune`` times the candidates on a
sample of the caller's queries with CUDA events, checks that every candidate
returns the same ids, and keeps the fastest.  Choices are cached per (GPU name, dim, adjacency row
stride, L rounded up to a power of two) in a JSON file, so ``apply`` can
reuse them without timing.
"""
from __future__ import annotations

import json
import os
import threading

import numpy as np

DEFAULT_CACHE = os.path.join(os.path.expanduser("~"), ".cache", "scattersearch_b200",
                             "tuning.json")
WPB_CANDIDATES = (1, 2, 4, 8)
# (teams per CTA, shared row stages) layouts tried besides one stage per team
SHARED_CANDIDATES = ((2, 1), (4, 2), (4, 3), (8, 3), (8, 4), (8, 5))
# rows per row stage tried with one stage per team (16 = the default; 24 takes
# most hops' fresh rows in one copy round trip, at fewer teams per SM)
STAGE_ROWS_CANDIDATES = (16, 12, 24)
# the fastest layouts with visited marks are timed again without them
MARKS_OFF_TOP = 6
_lock = threading.Lock()


def l_bucket(L: int) -> int:
    """L rounded up to a power of two (tuning keys cover L ranges)."""
    b = 1
    while b < L:
        b <<= 1
    return b


def hash_candidates(L: int):
    """Visited-table sizes worth timing for beam width L."""
    lo = 1024
    hi = max(lo, min(65536, l_bucket(L) * 32))
    out, c = [], lo
    while c <= hi:
        out.append(c)
        c <<= 1
    return out


def tuning_key(gpu: str, dim: int, rstride: int, L: int) -> str:
    return f"{gpu}|dim={dim}|rstride={rstride}|L<={l_bucket(L)}"


def load_cache(path: str = DEFAULT_CACHE) -> dict:
    try:
        with open(path) as f:
            data = json.load(f)
        return data if isinstance(data, dict) else {}
    except (OSError, ValueError):
        return {}


def save_choice(key: str, choice: dict, path: str = DEFAULT_CACHE) -> None:
    with _lock:
        data = load_cache(path)
        data[key] = choice
        os.makedirs(os.path.dirname(path) or ".", exist_ok=True)
        tmp = path + ".tmp"
        with open(tmp, "w") as f:
            json.dump(data, f, indent=1, sort_keys=True)
        os.replace(tmp, path)


def _gpu_name(device) -> str:
    import torch
    return torch.cuda.get_device_name(device)


def apply(index, L: int, path: str = DEFAULT_CACHE, device=None) -> dict | None:
    """Sets the cached choice for (this GPU, index shape, L) on ``index``;
    returns it, or None (and leaves the automatic setting) when none is
    cached."""
    key = tuning_key(_gpu_name(device), index.dimension, index.rstride, L)
    choice = load_cache(path).get(key)
    if choice:
        index.set_tuning(int(choice["warps_per_block"]), int(choice["hash_cap"]), 0,
                         int(choice.get("shared_stages", 0)), int(choice.get("stage_rows", 0)))
        index.set_visited_marks(int(choice.get("visited_marks", 0)))
    return choice


def autotune(index, queries, K: int, L: int, reps: int = 3, path: str | None = DEFAULT_CACHE,
             device=None, wpb_candidates=WPB_CANDIDATES, hash_caps=None, Ks=None, Ls=None,
             out_off=None, shared_candidates=SHARED_CANDIDATES,
             stage_rows_candidates=STAGE_ROWS_CANDIDATES, marks_off_top=MARKS_OFF_TOP) -> dict:
    """Times every (warps_per_block, shared_stages, stage_rows, hash_cap)
    candidate -- each of ``wpb_candidates`` with a stage per team of each of
    ``stage_rows_candidates`` rows, and each pair of ``shared_candidates``
    with 16-row stages -- with visited marks, then the ``marks_off_top``
    fastest of them without (``visited_marks`` 1), on ``queries`` (a
    CUDA tensor, nq x dim) and sets the fastest on ``index``.  Raises if two
    candidates return different ids.  Returns the choice with the timing
    table; stores it in the cache at ``path`` (None: no cache).

    For a batch with per-query K and L, pass the device arrays ``Ks``, ``Ls``
    and ``out_off`` (as for ``search_batch_device``); ``K`` is then the total
    number of result slots and ``L`` the largest L of the batch."""
    import torch
    nq = int(queries.shape[0])
    dev = queries.device
    uneven = Ks is not None
    ids = torch.empty((K,) if uneven else (nq, K), dtype=torch.int32, device=dev)
    stream = torch.cuda.current_stream(dev)

    def launch():
        if uneven:
            index.search_batch_device(queries, nq, ids, None, Ks=Ks, Ls=Ls, out_off=out_off,
                                      L_max=L, stream=stream.cuda_stream)
        else:
            index.search_batch_device(queries, nq, ids, None, K=K, L=L,
                                      stream=stream.cuda_stream)

    ref = None
    table = []

    def time_one(wpb, stages, rows, hc, marks):
        nonlocal ref
        index.set_tuning(wpb, hc, 0, stages, rows)
        index.set_visited_marks(marks)
        launch()
        stream.synchronize()
        got = ids.cpu().numpy()
        if ref is None:
            ref = got.copy()
        elif not np.array_equal(got, ref):
            raise RuntimeError(f"ids differ under warps_per_block={wpb}, "
                               f"shared_stages={stages}, stage_rows={rows}, hash_cap={hc}, "
                               f"visited_marks={marks}")
        times = []
        for _ in range(reps):
            a = torch.cuda.Event(enable_timing=True)
            b = torch.cuda.Event(enable_timing=True)
            a.record(stream)
            launch()
            b.record(stream)
            stream.synchronize()
            times.append(a.elapsed_time(b))
        table.append({"warps_per_block": wpb, "shared_stages": stages, "stage_rows": rows,
                      "hash_cap": hc, "visited_marks": marks, "ms": float(np.median(times))})

    layouts = [(w, 0, r) for r in (stage_rows_candidates or (16,)) for w in wpb_candidates]
    layouts += [(w, st, 16) for w, st in (shared_candidates or ())]
    for hc in (hash_caps or hash_candidates(L)):
        for wpb, stages, rows in layouts:
            time_one(wpb, stages, rows, hc, 0)
    for r in sorted(table, key=lambda r: r["ms"])[:max(0, marks_off_top)]:
        time_one(r["warps_per_block"], r["shared_stages"], r["stage_rows"], r["hash_cap"], 1)
    best = min(table, key=lambda r: r["ms"])
    index.set_tuning(best["warps_per_block"], best["hash_cap"], 0, best["shared_stages"],
                     best["stage_rows"])
    index.set_visited_marks(best["visited_marks"])
    choice = {"warps_per_block": best["warps_per_block"], "shared_stages": best["shared_stages"],
              "stage_rows": best["stage_rows"], "hash_cap": best["hash_cap"],
              "visited_marks": best["visited_marks"], "ms": best["ms"],
              "sample_queries": nq, "K": "per query" if uneven else K, "L": L}
    if path:
        save_choice(tuning_key(_gpu_name(device if device is not None else dev),
                               index.dimension, index.rstride, L), choice, path)
    return dict(choice, table=table)
