"""Seeded synthetic point clouds for the ridge-detection workloads.

The reference ships only unseeded generators (rd/cpu/samples_generator.hpp:42-200,
std::random_device) and names data files that are not in its repository, so every
workload here is regenerated from a numpy PCG64 stream with a fixed seed.  All
clouds are float32, ROW_MAJOR (point i at P[i*dim + d]) and come out in
generation order, which is the order the greedy choose visits them.

Workloads (sizes and parameters as the benchmark defines them):
  sine2d     N=20,000, t~U[0,10], p=(t, sin 2t) + N(0, 0.1^2) per coord,  r1=0.3,  r2=0.6
  helix3d    N=1,000,000, t~U[0,8pi], p=(cos t, sin t, 0.15 t) + N(0, 0.05^2), r1=0.15, r2=0.3
  spiral2d   N=10,000,000, 95% p=0.5 th (cos th, sin th) + N(0, 0.05^2), th~U[0,6pi];
             5% uniform in the bounding box of the spiral part; r1=0.2, r2=0.4, 64x64 tiles
  batch      4,096 clouds, N_c=round(exp(U[ln 1e3, ln 2e5])), even c sine2d / odd c helix3d,
             r1_c~U[0.1,0.3], r2_c=2 r1_c, cloud c seeded with SEED_BASE + c
"""
from __future__ import annotations

import math

import numpy as np

SEED_BASE = 0x5EED


def sine2d(n: int, seed: int = SEED_BASE, noise: float = 0.1) -> np.ndarray:
    rng = np.random.default_rng(seed)
    t = rng.uniform(0.0, 10.0, n)
    p = np.empty((n, 2), dtype=np.float64)
    p[:, 0] = t
    p[:, 1] = np.sin(2.0 * t)
    p += rng.normal(0.0, noise, (n, 2))
    return np.ascontiguousarray(p, dtype=np.float32)


def helix3d(n: int, seed: int = SEED_BASE, noise: float = 0.05) -> np.ndarray:
    rng = np.random.default_rng(seed)
    t = rng.uniform(0.0, 8.0 * math.pi, n)
    p = np.empty((n, 3), dtype=np.float64)
    p[:, 0] = np.cos(t)
    p[:, 1] = np.sin(t)
    p[:, 2] = 0.15 * t
    p += rng.normal(0.0, noise, (n, 3))
    return np.ascontiguousarray(p, dtype=np.float32)


def spiral2d(n: int, seed: int = SEED_BASE, noise: float = 0.05,
             clutter: float = 0.05) -> np.ndarray:
    rng = np.random.default_rng(seed)
    n_clut = int(round(n * clutter))
    n_sp = n - n_clut
    th = rng.uniform(0.0, 6.0 * math.pi, n_sp)
    sp = np.empty((n_sp, 2), dtype=np.float64)
    sp[:, 0] = 0.5 * th * np.cos(th)
    sp[:, 1] = 0.5 * th * np.sin(th)
    sp += rng.normal(0.0, noise, (n_sp, 2))
    lo = sp.min(axis=0)
    hi = sp.max(axis=0)
    cl = rng.uniform(lo, hi, (n_clut, 2))
    p = np.concatenate([sp, cl], axis=0)
    # interleave clutter with the curve so the visiting order is not blocked
    p = p[rng.permutation(n)]
    return np.ascontiguousarray(p, dtype=np.float32)


def ideal_spiral2d(n: int, seed: int = SEED_BASE) -> np.ndarray:
    """Noise-free points of the curve spiral2d samples, 0.5*theta*(cos, sin)
    for theta uniform in [0, 6*pi]: an ideal pattern for the quality metrics
    (the role of genSpiral2D with sigma = 0, rd/cpu/samples_generator.hpp:42)."""
    th = np.random.default_rng(seed).uniform(0.0, 6.0 * math.pi, n)
    return np.ascontiguousarray(np.stack([0.5 * th * np.cos(th), 0.5 * th * np.sin(th)], 1),
                                dtype=np.float32)


def ideal_helix3d(n: int, seed: int = SEED_BASE) -> np.ndarray:
    """Noise-free points of the curve helix3d samples, (cos t, sin t, 0.15 t)
    for t uniform in [0, 8*pi]."""
    t = np.random.default_rng(seed).uniform(0.0, 8.0 * math.pi, n)
    return np.ascontiguousarray(np.stack([np.cos(t), np.sin(t), 0.15 * t], 1), dtype=np.float32)


def batch_spec(n_clouds: int = 4096, seed_base: int = SEED_BASE,
               n_min: int = 1000, n_max: int = 200_000):
    """Per-cloud (n, dim, r1, r2, seed) of the batched workload."""
    spec = []
    for c in range(n_clouds):
        rng = np.random.default_rng(seed_base + c)
        n = int(round(math.exp(rng.uniform(math.log(n_min), math.log(n_max)))))
        r1 = float(np.float32(rng.uniform(0.1, 0.3)))
        r2 = float(np.float32(2.0 * np.float32(r1)))
        dim = 2 if c % 2 == 0 else 3
        spec.append((n, dim, r1, r2, seed_base + 1_000_003 * (c + 1)))
    return spec


def batch_cloud(n: int, dim: int, seed: int) -> np.ndarray:
    return sine2d(n, seed) if dim == 2 else helix3d(n, seed)


WORKLOADS = {
    "sine2d_20k": dict(gen=sine2d, n=20_000, dim=2, r1=0.3, r2=0.6),
    "helix3d_1m": dict(gen=helix3d, n=1_000_000, dim=3, r1=0.15, r2=0.3),
    "spiral2d_10m": dict(gen=spiral2d, n=10_000_000, dim=2, r1=0.2, r2=0.4,
                         tiles=(64, 64)),
}
