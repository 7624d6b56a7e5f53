"""Seeded synthetic workloads standing in for the reference's datasets.

The reference benchmarks on external files (Glove-200, SIFT-like, DEEP, ...)
that are not available here.  These generators produce inputs with the
shapes, sizes and value distributions of the five benchmark configurations;
no item of any public dataset is reproduced.  All draws use
``numpy.random.default_rng`` with fixed seeds: mixture parameters 3000+cfg,
base vectors 1000+cfg, queries 2000+cfg.

  cfg 1  100k x 200, 10-component Gaussian mixture (means N(0,1), sd 0.3),
         L2-normalised; 1k queries; L2, K=10, L=100
  cfg 2  1M x 128, clip(round(Gamma(0.8, 40) * s_d), 0, 255), s_d ~ U(0.5,1.5)
         per dimension; 10k queries; L2, K=10, L in {64,128,256}
  cfg 3  1.2M x 200, 50-component mixture, log-normal(0, 0.5) norm scale,
         unit-normalised (angular); inner product, K=100, L in {200,400}
  cfg 4  5M x 96, 100-component mixture, unit-normalised; 100k queries with
         K in {1,10,100}, L ~ U[32,512]
  cfg 5  cfg 3's index under Poisson arrivals
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

L2, IP = 0, 1


@dataclass
class Workload:
    name: str
    base: np.ndarray
    queries: np.ndarray
    metric: int
    K: int
    L_list: list = field(default_factory=list)
    graph_R: int = 32
    graph_knn: int = 64


def _mixture(rng, means, sd, n, chunk=1 << 18):
    """n draws from an isotropic Gaussian mixture with equal weights."""
    c, d = means.shape
    out = np.empty((n, d), dtype=np.float32)
    for s in range(0, n, chunk):
        e = min(n, s + chunk)
        comp = rng.integers(0, c, size=e - s)
        out[s:e] = means[comp] + sd * rng.standard_normal((e - s, d), dtype=np.float32)
    return out


def _normalise(x):
    n = np.linalg.norm(x, axis=1, keepdims=True)
    n[n == 0] = 1.0
    x /= n
    return x


def gaussian_mixture(n, dim, components, sd, seed, mix_seed, lognormal_sigma=0.0):
    mrng = np.random.default_rng(mix_seed)
    means = mrng.standard_normal((components, dim), dtype=np.float32)
    rng = np.random.default_rng(seed)
    x = _mixture(rng, means, sd, n)
    if lognormal_sigma > 0:
        x *= rng.lognormal(0.0, lognormal_sigma, size=(n, 1)).astype(np.float32)
    return _normalise(x)


def gamma_uint8(n, dim, seed, mix_seed):
    scale = np.random.default_rng(mix_seed).uniform(0.5, 1.5, size=dim).astype(np.float32)
    rng = np.random.default_rng(seed)
    out = np.empty((n, dim), dtype=np.float32)
    chunk = 1 << 18
    for s in range(0, n, chunk):
        e = min(n, s + chunk)
        g = rng.gamma(0.8, 40.0, size=(e - s, dim)).astype(np.float32) * scale
        out[s:e] = np.clip(np.round(g), 0, 255)
    return out


def config(cfg: int, scale: float = 1.0, n_queries: int | None = None) -> Workload:
    """Workload of configuration ``cfg`` (1..5).  ``scale`` shrinks the base
    size (tests use small fractions); the distributions are unchanged."""
    def nb(full):
        return max(1000, int(full * scale))

    if cfg == 1:
        n, nq = nb(100_000), n_queries or 1000
        gen = lambda cnt, seed: gaussian_mixture(cnt, 200, 10, 0.3, seed, 3001)
        return Workload("cfg1-100kx200-l2", gen(n, 1001), gen(nq, 2001), L2, 10, [100], 32, 64)
    if cfg == 2:
        n, nq = nb(1_000_000), n_queries or 10_000
        return Workload("cfg2-1Mx128-l2-uint8", gamma_uint8(n, 128, 1002, 3002),
                        gamma_uint8(nq, 128, 2002, 3002), L2, 10, [64, 128, 256], 64, 100)
    if cfg in (3, 5):
        n, nq = nb(1_200_000), n_queries or 10_000
        gen = lambda cnt, seed: gaussian_mixture(cnt, 200, 50, 0.3, seed, 3003, 0.5)
        return Workload("cfg3-1.2Mx200-ip" if cfg == 3 else "cfg5-serving-1.2Mx200-ip",
                        gen(n, 1003), gen(nq, 2003), IP, 100, [200, 400], 32, 64)
    if cfg == 4:
        n, nq = nb(5_000_000), n_queries or 100_000
        gen = lambda cnt, seed: gaussian_mixture(cnt, 96, 100, 0.3, seed, 3004)
        return Workload("cfg4-5Mx96-ip-uneven", gen(n, 1004), gen(nq, 2004), IP, 100, [], 32, 64)
    raise ValueError(f"unknown config {cfg}")


def uneven_k_l(nq: int, seed: int = 4004, k_choices=(1, 10, 100), l_range=(32, 512)):
    """Per-query K in k_choices and L ~ U[l_range] with L >= K (config 4)."""
    rng = np.random.default_rng(seed)
    Ks = rng.choice(np.array(k_choices, dtype=np.int32), size=nq)
    Ls = rng.integers(l_range[0], l_range[1] + 1, size=nq).astype(np.int32)
    return Ks.astype(np.int32), np.maximum(Ls, Ks).astype(np.int32)
