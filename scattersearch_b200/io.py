"""Readers and writers for the reference's on-disk formats (numpy, host side).

* ``.fbin``  ``u32 num, u32 dim, num*dim f32``   -- load_fbin, src/util.cpp:40-70
* ground truth ``u32 nq, u32 K, nq*K u32``       -- load_groundtruth, src/util.cpp:72-93
* ``.fvecs`` per row ``i32 dim, dim f32``         -- load_fvecs, src/util.cpp:6-38
* ``.nsg``   ``u32 width, u32 ep``, then per node ``u32 k, k u32``
                                                  -- ANNSearch::LoadGraph, src/annsearch.cpp:64-80

Graphs are handled as ``n x R`` uint32 tables padded with 0xFFFFFFFF, the
layout the device kernels use.  The C ABI has native loaders for the same
formats (ss_load_fbin, ss_load_groundtruth, ss_load_graph); these are for
tools and tests.

Data tools (the reference's scripts/splitfbin.py and scripts/hdf5tofbin.py):
``split_fbin`` keeps the last vectors of an ``.fbin`` file as the query set
and the rest as the base set; ``ann_benchmarks_to_fbin`` writes an
ann-benchmarks style (train, test, neighbors) triple as base and query
``.fbin`` files and a ground-truth file, and ``hdf5_to_fbin`` reads that
triple from an HDF5 file.  ``python -m scattersearch_b200.io`` runs either
from the command line.
"""
from __future__ import annotations

import numpy as np

NONE_ID = 0xFFFFFFFF


class FormatError(ValueError):
    pass


def write_fbin(path: str, data) -> None:
    a = np.ascontiguousarray(data, dtype=np.float32)
    if a.ndim != 2:
        raise ValueError("fbin data must be 2-D")
    with open(path, "wb") as f:
        np.array(a.shape, dtype=np.uint32).tofile(f)
        a.tofile(f)


def load_fbin(path: str) -> np.ndarray:
    with open(path, "rb") as f:
        hdr = np.fromfile(f, dtype=np.uint32, count=2)
        if hdr.size != 2:
            raise FormatError(f"{path}: missing fbin header")
        n, d = int(hdr[0]), int(hdr[1])
        a = np.fromfile(f, dtype=np.float32, count=n * d)
    if a.size != n * d:
        raise FormatError(f"{path}: expected {n}x{d} floats, found {a.size}")
    return a.reshape(n, d)


def write_groundtruth(path: str, ids) -> None:
    a = np.ascontiguousarray(ids, dtype=np.uint32)
    with open(path, "wb") as f:
        np.array(a.shape, dtype=np.uint32).tofile(f)
        a.tofile(f)


def load_groundtruth(path: str) -> np.ndarray:
    with open(path, "rb") as f:
        hdr = np.fromfile(f, dtype=np.uint32, count=2)
        if hdr.size != 2:
            raise FormatError(f"{path}: missing ground-truth header")
        nq, k = int(hdr[0]), int(hdr[1])
        a = np.fromfile(f, dtype=np.uint32, count=nq * k)
    if a.size != nq * k:
        raise FormatError(f"{path}: expected {nq}x{k} ids, found {a.size}")
    return a.reshape(nq, k)


def load_fvecs(path: str) -> np.ndarray:
    raw = np.fromfile(path, dtype=np.int32)
    if raw.size == 0:
        return np.zeros((0, 0), dtype=np.float32)
    d = int(raw[0])
    if raw.size % (d + 1):
        raise FormatError(f"{path}: size is not a multiple of the row length")
    return raw.reshape(-1, d + 1)[:, 1:].copy().view(np.float32)


def write_nsg(path: str, adj, ep: int, width: int | None = None) -> None:
    a = np.asarray(adj, dtype=np.uint32)
    deg = (a != NONE_ID).sum(axis=1)
    with open(path, "wb") as f:
        np.array([int(width if width is not None else deg.max(initial=0)), int(ep)],
                 dtype=np.uint32).tofile(f)
        for i in range(a.shape[0]):
            row = a[i, :deg[i]]
            np.array([row.size], dtype=np.uint32).tofile(f)
            row.tofile(f)


def read_nsg(path: str):
    """Returns (adj n x R padded with NONE_ID, entry point, width field)."""
    raw = np.fromfile(path, dtype=np.uint32)
    if raw.size < 2:
        raise FormatError(f"{path}: missing NSG header")
    width, ep = int(raw[0]), int(raw[1])
    rows = []
    pos = 2
    while pos < raw.size:
        k = int(raw[pos])
        if pos + 1 + k > raw.size:
            raise FormatError(f"{path}: truncated record for node {len(rows)}")
        rows.append(raw[pos + 1:pos + 1 + k])
        pos += 1 + k
    R = max((r.size for r in rows), default=0)
    adj = np.full((len(rows), max(R, 1)), NONE_ID, dtype=np.uint32)
    for i, r in enumerate(rows):
        adj[i, :r.size] = r
    return adj, ep, width


def split_fbin(path: str, num_queries: int = 1000, base_out: str = "base.fbin",
               query_out: str = "query.fbin"):
    """Splits an ``.fbin`` file: its last ``num_queries`` vectors go to
    ``query_out`` and the others, in order, to ``base_out`` (the split of
    scripts/splitfbin.py).  The input is memory-mapped, so files larger
    than host memory work.  Returns (n_base, n_query, dim)."""
    with open(path, "rb") as f:
        hdr = np.fromfile(f, dtype=np.uint32, count=2)
    if hdr.size != 2:
        raise FormatError(f"{path}: missing fbin header")
    n, d = int(hdr[0]), int(hdr[1])
    if num_queries < 0 or num_queries > n:
        raise ValueError(f"{path} holds {n} vectors; cannot split off {num_queries} queries")
    data = np.memmap(path, dtype=np.float32, mode="r", offset=8, shape=(n, d))
    n_base = n - num_queries
    for out, part in ((base_out, data[:n_base]), (query_out, data[n_base:])):
        with open(out, "wb") as f:
            np.array(part.shape, dtype=np.uint32).tofile(f)
            step = max(1, (1 << 26) // max(1, 4 * d))  # about 64 MB per write
            for s in range(0, part.shape[0], step):
                np.ascontiguousarray(part[s:s + step]).tofile(f)
    del data
    return n_base, num_queries, d


def ann_benchmarks_to_fbin(train, test, neighbors, base_out: str, query_out: str, gt_out: str,
                           k: int | None = None) -> None:
    """Writes base (``train``) and query (``test``) vectors as float32
    ``.fbin`` files and the first ``k`` (default: all) columns of
    ``neighbors`` as a ground-truth file (the conversion of
    scripts/hdf5tofbin.py; float64 inputs are converted to float32, which
    the ``.fbin`` format holds)."""
    train = np.asarray(train)
    test = np.asarray(test)
    nbr = np.asarray(neighbors)
    if train.ndim != 2 or test.ndim != 2 or train.shape[1] != test.shape[1]:
        raise ValueError("train and test must be 2-D with the same dimension")
    if nbr.ndim != 2 or nbr.shape[0] != test.shape[0]:
        raise ValueError("neighbors must hold one row per test vector")
    if nbr.size and (nbr.min() < 0 or nbr.max() >= train.shape[0]):
        raise ValueError("neighbors hold ids outside the train set")
    write_fbin(base_out, train.astype(np.float32, copy=False))
    write_fbin(query_out, test.astype(np.float32, copy=False))
    write_groundtruth(gt_out, nbr[:, :k] if k else nbr)


def hdf5_to_fbin(path: str, base_out: str, query_out: str, gt_out: str,
                 k: int | None = None) -> None:
    """``ann_benchmarks_to_fbin`` on the ``train``, ``test`` and ``neighbors``
    datasets of an HDF5 file (needs h5py)."""
    try:
        import h5py
    except ImportError as e:  # pragma: no cover - depends on the environment
        raise ImportError("hdf5_to_fbin needs h5py, which is not installed") from e
    with h5py.File(path, "r") as f:
        ann_benchmarks_to_fbin(f["train"][:], f["test"][:], f["neighbors"][:], base_out,
                               query_out, gt_out, k)


def main(argv=None) -> int:
    import argparse
    ap = argparse.ArgumentParser(prog="python -m scattersearch_b200.io",
                                 description="Data tools for the .fbin / ground-truth formats.")
    sub = ap.add_subparsers(dest="cmd", required=True)
    sp = sub.add_parser("split-fbin", help="split the last vectors of an .fbin off as queries")
    sp.add_argument("path")
    sp.add_argument("--num-queries", type=int, default=1000)
    sp.add_argument("--base-out", default="base.fbin")
    sp.add_argument("--query-out", default="query.fbin")
    hp = sub.add_parser("hdf5-to-fbin", help="convert an ann-benchmarks HDF5 file")
    hp.add_argument("path")
    hp.add_argument("--base-out", default="base.fbin")
    hp.add_argument("--query-out", default="query.fbin")
    hp.add_argument("--gt-out", default="groundtruth.bin")
    hp.add_argument("--k", type=int, default=None)
    args = ap.parse_args(argv)
    if args.cmd == "split-fbin":
        nb, nq, d = split_fbin(args.path, args.num_queries, args.base_out, args.query_out)
        print(f"{args.base_out}: {nb} x {d}; {args.query_out}: {nq} x {d}")
    else:
        hdf5_to_fbin(args.path, args.base_out, args.query_out, args.gt_out, args.k)
        print(f"wrote {args.base_out}, {args.query_out}, {args.gt_out}")
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
