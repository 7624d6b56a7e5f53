"""NSG-style proximity-graph builder (kNN -> MRNG prune -> reverse edges ->
re-prune -> connectivity repair), in torch on any device.

The reference ships no graph builder: its ``.nsg`` inputs come from outside
the repository (ANNSearch::LoadGraph, src/annsearch.cpp:64-80, only reads
them).  The benchmark configurations call for "exact k-NN followed by MRNG
pruning to out-degree <= R, entry point = medoid"; this module builds such
graphs so the search has inputs of the right kind.  It is setup code, not the
timed path.

Edge selection is the MRNG rule: candidates of node p are taken in ascending
distance and a candidate c is kept unless an already kept neighbour r is
closer to c than p is (d(r, c) < d(p, c)).  Reverse edges are then offered to
their targets and every node is pruned again, and finally nodes unreachable
from the entry point are linked from their nearest reachable neighbour.
Distances are squared L2 on the stored vectors (for unit-normalised data this
orders neighbours exactly as inner product does).
"""
from __future__ import annotations

import numpy as np
import torch

NONE_ID = 0xFFFFFFFF


def _pick_chunk(n: int, bytes_per_row: int, budget: float) -> int:
    return int(max(64, min(16384, budget // max(1, bytes_per_row))))


@torch.no_grad()
def knn(X: torch.Tensor, k: int, chunk: int | None = None, budget_bytes: float = 6e9):
    """Exact k nearest neighbours of every row of X among the rows of X,
    excluding the row itself.  Returns (ids int64 [n,k], sq. dists [n,k])."""
    n = X.shape[0]
    xx = (X * X).sum(1)
    chunk = chunk or _pick_chunk(n, 4 * n, budget_bytes)
    out_i = torch.empty((n, k), dtype=torch.int64, device=X.device)
    out_d = torch.empty((n, k), dtype=torch.float32, device=X.device)
    for s in range(0, n, chunk):
        e = min(n, s + chunk)
        D = torch.addmm(xx[None, :], X[s:e], X.T, beta=1.0, alpha=-2.0)
        D += xx[s:e, None]
        D[torch.arange(e - s, device=X.device), torch.arange(s, e, device=X.device)] = float("inf")
        d, i = torch.topk(D, k, dim=1, largest=False, sorted=True)
        out_i[s:e] = i
        out_d[s:e] = d.clamp_min_(0)
        del D
    return out_i, out_d


@torch.no_grad()
def knn_tensor_cores(X: torch.Tensor, k: int, chunk: int = 1 << 18):
    """Exact k nearest neighbours of every row of X among the rows of X
    (squared L2, ties by smaller id), excluding the row itself, from the
    library's tensor-core brute force (ss_bruteforce_device) on X's CUDA
    device.  Returns (ids int64 [n,k], sq. dists [n,k]) like ``knn``."""
    from .annsearch import ANNSearch
    n, dim = X.shape
    if k + 1 > 112:
        raise ValueError("the brute force returns at most 112 neighbours")
    X = X.contiguous()
    dev = X.device.index if X.device.index is not None else -1
    idx = ANNSearch(dim, n, X, 0, device=dev, base_on_device=True)
    out_i = torch.empty((n, k), dtype=torch.int64, device=X.device)
    out_d = torch.empty((n, k), dtype=torch.float32, device=X.device)
    ids = torch.empty((min(chunk, n), k + 1), dtype=torch.int32, device=X.device)
    dists = torch.empty((min(chunk, n), k + 1), dtype=torch.float32, device=X.device)
    stream = torch.cuda.current_stream(X.device).cuda_stream
    try:
        for s in range(0, n, chunk):
            e = min(n, s + chunk)
            idx.bruteforce_device(X[s:e], e - s, k + 1, ids, dists, stream=stream)
            got = ids[:e - s].to(torch.int64) & 0xFFFFFFFF
            rows = torch.arange(s, e, device=X.device)
            # drop the row itself; when k+1 exact duplicates of it with smaller
            # ids push it out of the list, drop the last entry instead
            drop = got == rows[:, None]
            drop[~drop.any(1), -1] = True
            out_i[s:e] = got[~drop].view(e - s, k)
            out_d[s:e] = dists[:e - s][~drop].view(e - s, k)
        torch.cuda.synchronize(X.device)
    finally:
        idx.close()
    return out_i, out_d


@torch.no_grad()
def bruteforce(X: torch.Tensor, Q: torch.Tensor, k: int, metric: int, chunk: int | None = None,
               budget_bytes: float = 6e9, exact_dtype=torch.float64):
    """Exact top-k of Q against X: float32 candidate scan, then the top
    candidates re-ranked in float64.  metric 0: squared L2; 1: -inner product
    (the reference's sign, src/distance.cpp:148).  Returns (ids, dists)."""
    n = X.shape[0]
    kk = min(n, max(k * 2, k + 16))
    xx = (X * X).sum(1)
    chunk = chunk or _pick_chunk(n, 4 * n, budget_bytes)
    ids = torch.empty((Q.shape[0], k), dtype=torch.int64, device=X.device)
    dists = torch.empty((Q.shape[0], k), dtype=exact_dtype, device=X.device)
    for s in range(0, Q.shape[0], chunk):
        e = min(Q.shape[0], s + chunk)
        q = Q[s:e]
        if metric == 0:
            D = torch.addmm(xx[None, :], q, X.T, beta=1.0, alpha=-2.0)
        else:
            D = -(q @ X.T)
        _, cand = torch.topk(D, kk, dim=1, largest=False, sorted=False)
        del D
        V = X[cand].to(exact_dtype)
        qd = q.to(exact_dtype)[:, None, :]
        if metric == 0:
            ex = ((V - qd) ** 2).sum(-1)
        else:
            ex = -(V * qd).sum(-1)
        # stable order: distance, then id
        order = torch.argsort(cand, dim=1)
        cand = torch.gather(cand, 1, order)
        ex = torch.gather(ex, 1, order)
        d2, o2 = torch.sort(ex, dim=1, stable=True)
        ids[s:e] = torch.gather(cand, 1, o2[:, :k])
        dists[s:e] = d2[:, :k]
    return ids, dists


@torch.no_grad()
def mrng_prune(X: torch.Tensor, cand: torch.Tensor, cand_d: torch.Tensor, R: int,
               budget_bytes: float = 4e9):
    """MRNG selection of at most R neighbours per node from candidate lists
    sorted by ascending distance (-1 marks an empty slot)."""
    n, C = cand.shape
    d = X.shape[1]
    out = torch.full((n, R), -1, dtype=torch.int64, device=X.device)
    chunk = _pick_chunk(n, 4 * C * (d + C) * 2, budget_bytes)
    for s in range(0, n, chunk):
        e = min(n, s + chunk)
        ci = cand[s:e]
        cd = cand_d[s:e]
        valid = ci >= 0
        V = X[ci.clamp_min(0)]
        vv = (V * V).sum(-1)
        P = torch.baddbmm(vv[:, :, None] + vv[:, None, :], V, V.transpose(1, 2), beta=1.0,
                          alpha=-2.0)
        del V
        B = e - s
        sel = torch.zeros((B, C), dtype=torch.bool, device=X.device)
        cnt = torch.zeros(B, dtype=torch.int64, device=X.device)
        for j in range(C):
            conflict = (sel & (P[:, :, j] < cd[:, j:j + 1])).any(1)
            keep = valid[:, j] & ~conflict & (cnt < R)
            sel[:, j] = keep
            cnt += keep
        # selected ids in candidate order
        rank = torch.cumsum(sel.to(torch.int64), dim=1) - 1
        rows = torch.arange(B, device=X.device)[:, None].expand(B, C)
        m = sel & (rank < R)
        blk = torch.full((B, R), -1, dtype=torch.int64, device=X.device)
        blk[rows[m], rank[m]] = ci[m]
        out[s:e] = blk
    return out


@torch.no_grad()
def _pair_sqdist(X, a, b, chunk=1 << 22):
    out = torch.empty(a.shape[0], dtype=torch.float32, device=X.device)
    for s in range(0, a.shape[0], chunk):
        e = min(a.shape[0], s + chunk)
        out[s:e] = ((X[a[s:e]] - X[b[s:e]]) ** 2).sum(1)
    return out


@torch.no_grad()
def add_reverse_edges(X: torch.Tensor, adj: torch.Tensor, R: int, rev_cap: int | None = None):
    """Offers every edge p->q back to q (NSG's inter-insert) and prunes each
    node's union of forward and reverse candidates to R with MRNG."""
    n = adj.shape[0]
    rev_cap = rev_cap or R
    valid = adj >= 0
    src = torch.arange(n, device=X.device)[:, None].expand_as(adj)[valid]
    dst = adj[valid]
    ed = _pair_sqdist(X, src, dst)
    # group by target, nearest sources first
    o = torch.argsort(ed, stable=True)
    src, dst, ed = src[o], dst[o], ed[o]
    o = torch.argsort(dst, stable=True)
    src, dst, ed = src[o], dst[o], ed[o]
    counts = torch.bincount(dst, minlength=n)
    start = torch.cumsum(counts, 0) - counts
    pos = torch.arange(dst.shape[0], device=X.device) - start[dst]
    keep = pos < rev_cap
    rev = torch.full((n, rev_cap), -1, dtype=torch.int64, device=X.device)
    rev_d = torch.full((n, rev_cap), float("inf"), device=X.device)
    rev[dst[keep], pos[keep]] = src[keep]
    rev_d[dst[keep], pos[keep]] = ed[keep]
    # forward distances
    fwd_d = torch.full(adj.shape, float("inf"), device=X.device)
    rows = torch.arange(n, device=X.device)[:, None].expand_as(adj)
    fwd_d[valid] = _pair_sqdist(X, rows[valid], adj[valid])
    cand = torch.cat([adj, rev], 1)
    cd = torch.cat([fwd_d, rev_d], 1)
    # sort by (distance, id); drop duplicates (same pair -> same distance)
    big = torch.where(cand >= 0, cand, torch.full_like(cand, n))
    o = torch.argsort(big, dim=1, stable=True)
    cand, cd = torch.gather(cand, 1, o), torch.gather(cd, 1, o)
    o = torch.argsort(cd, dim=1, stable=True)
    cand, cd = torch.gather(cand, 1, o), torch.gather(cd, 1, o)
    dup = torch.zeros_like(cand, dtype=torch.bool)
    dup[:, 1:] = (cand[:, 1:] == cand[:, :-1]) & (cand[:, 1:] >= 0)
    cand = torch.where(dup, torch.full_like(cand, -1), cand)
    cd = torch.where(dup, torch.full_like(cd, float("inf")), cd)
    o = torch.argsort(cd, dim=1, stable=True)
    cand, cd = torch.gather(cand, 1, o), torch.gather(cd, 1, o)
    return mrng_prune(X, cand, cd, R)


def medoid(X: torch.Tensor) -> int:
    """Index of the row nearest (squared L2) to the centroid."""
    c = X.mean(0, keepdim=True)
    return int(((X - c) ** 2).sum(1).argmin().item())


def _csr(adj_np: np.ndarray):
    import scipy.sparse as sp
    n, R = adj_np.shape
    valid = adj_np >= 0
    rows = np.repeat(np.arange(n), R)[valid.reshape(-1)]
    cols = adj_np[valid]
    return sp.csr_matrix((np.ones(rows.size, dtype=np.int8), (rows, cols)), shape=(n, n))


def _reach_from(adj_np: np.ndarray, src: int) -> np.ndarray:
    from scipy.sparse.csgraph import breadth_first_order
    return breadth_first_order(_csr(adj_np), src, directed=True, return_predecessors=False)


@torch.no_grad()
def link_components(adj: np.ndarray, ep: int, X: torch.Tensor, long_links: int = 16,
                    seed: int = 7):
    """Adds long-range edges between weakly connected components.

    k-NN candidates never leave a well-separated cluster, so a pruned k-NN
    graph over clustered data splits into one component per cluster, and the
    similarity of a query to any other cluster carries no direction for a
    greedy search to follow.  Every component gets a representative (its
    member nearest to its centroid), and every node fills up to `long_links`
    of its free slots with edges to representatives of other components,
    chosen by a seeded random rotation; the entry point fills all its free
    slots.  Pruned neighbours are never displaced.  Expanding a handful of
    nodes then exposes the representative of every cluster, and the one the
    query belongs to stands out by distance."""
    from scipy.sparse.csgraph import connected_components
    adj = adj.copy()
    n, R = adj.shape
    ncomp, label = connected_components(_csr(adj), directed=True, connection="weak")
    if ncomp <= 1:
        return adj
    lab = torch.as_tensor(label, device=X.device, dtype=torch.int64)
    cnt = torch.bincount(lab, minlength=ncomp).to(torch.float32)
    cent = torch.zeros((ncomp, X.shape[1]), device=X.device).index_add_(0, lab, X)
    cent /= cnt[:, None]
    dist_to_cent = ((X - cent[lab]) ** 2).sum(1)
    best = torch.full((ncomp,), float("inf"), device=X.device).scatter_reduce(
        0, lab, dist_to_cent, reduce="amin")
    rep = np.full(ncomp, -1, dtype=np.int64)
    for i in torch.nonzero(dist_to_cent <= best[lab]).flatten().cpu().numpy():
        if rep[label[i]] < 0:
            rep[label[i]] = i
    deg = (adj >= 0).sum(1)
    rng = np.random.default_rng(seed)
    start = rng.integers(0, ncomp, size=n)
    want = np.minimum(R - deg, long_links)
    want[ep] = R - deg[ep]
    want = np.minimum(want, ncomp - 1)
    for j in range(int(want.max(initial=0))):
        # j-th long link: the (start + j)-th component after the node's own,
        # so the ncomp-1 picks of a node are distinct and never its own
        c = (label + 1 + (start + j) % (ncomp - 1)) % ncomp
        sel = np.flatnonzero(want > j)
        adj[sel, deg[sel]] = rep[c[sel]]
        deg[sel] += 1
    return adj


@torch.no_grad()
def repair_connectivity(adj: np.ndarray, knn_ids: np.ndarray, ep: int, X: torch.Tensor):
    """Makes every node reachable from ep.  Unreachable nodes are visited in
    id order; each one still unreached gets one in-edge from a reachable node
    with a free slot -- its nearest reachable k-NN neighbour when there is
    one, else the nearest such node by brute force -- and everything it
    reaches is marked reached (an incremental search over unreached nodes
    only).  Existing edges are never replaced."""
    adj = adj.copy()
    n, R = adj.shape
    seen = np.zeros(n, dtype=bool)
    seen[_reach_from(adj, ep)] = True
    if seen.all():
        return adj
    deg = (adj >= 0).sum(1)
    for u in np.flatnonzero(~seen):
        if seen[u]:
            continue
        nb = knn_ids[u]
        ok = nb[seen[nb] & (deg[nb] < R)]
        if ok.size:
            v = int(ok[0])
        else:
            d = ((X - X[u]) ** 2).sum(1)
            mask = torch.as_tensor(seen & (deg < R), device=X.device)
            d = torch.where(mask, d, torch.full_like(d, float("inf")))
            v = int(d.argmin().item())
            if not bool(mask[v]):
                raise RuntimeError("graph repair: no reachable node has a free slot")
        adj[v, deg[v]] = u
        deg[v] += 1
        seen[u] = True
        stack = [int(u)]
        while stack:
            x = stack.pop()
            for y in adj[x, :deg[x]]:
                if not seen[y]:
                    seen[y] = True
                    stack.append(int(y))
    return adj


@torch.no_grad()
def build_graph(X, R: int = 32, knn_k: int = 64, device: str | torch.device | None = None,
                reverse: bool = True, repair: bool = True, knn_budget_bytes: float = 6e9,
                knn_backend: str = "torch"):
    """Builds an out-degree <= R graph over X (n x d float32, numpy or torch).
    ``knn_backend``: "torch" (FP32 matmul + top-k, any device; its
    ``knn_budget_bytes`` bounds one distance block) or "bruteforce" (the
    library's exact tensor-core k-NN, CUDA only).
    Returns (adj uint32 n x R padded with 0xFFFFFFFF, entry point)."""
    dev = torch.device(device) if device is not None else (
        torch.device("cuda") if torch.cuda.is_available() else torch.device("cpu"))
    Xt = torch.as_tensor(np.asarray(X, dtype=np.float32) if not torch.is_tensor(X) else X)
    Xt = Xt.to(dev, dtype=torch.float32).contiguous()
    n = Xt.shape[0]
    k = min(knn_k, n - 1)
    if knn_backend == "bruteforce":
        ids, d = knn_tensor_cores(Xt, k)
    elif knn_backend == "torch":
        ids, d = knn(Xt, k, budget_bytes=knn_budget_bytes)
    else:
        raise ValueError(f"unknown k-NN backend {knn_backend!r}")
    adj = mrng_prune(Xt, ids, d, R)
    if reverse:
        adj = add_reverse_edges(Xt, adj, R)
    ep = medoid(Xt)
    adj_np = adj.cpu().numpy()
    if repair:
        adj_np = link_components(adj_np, ep, Xt)
        adj_np = repair_connectivity(adj_np, ids.cpu().numpy(), ep, Xt)
    out = np.where(adj_np >= 0, adj_np, NONE_ID).astype(np.uint32)
    # valid ids must form a prefix of each row
    order = np.argsort(out == NONE_ID, axis=1, kind="stable")
    out = np.take_along_axis(out, order, axis=1)
    return out, ep
