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
