"""Full-size golden results from the reference's own serial CPU code.

The workloads the benchmark measures are too large to store as clouds (the 10M
spiral alone is 80 MB), so these fixtures store how to regenerate the cloud
(generator, size, seed), a SHA-256 of the regenerated float32 bytes (to catch a
generator that drifted), and the reference's outputs:

  full_helix3d_1m.npz        brute force, helix N = 1,000,000, r1 = 0.15, r2 = 0.3:
                             the chosen set right after choose, the chosen set after
                             each of the first five evolve passes, and the final ridge
  full_spiral2d_10m_tiled.npz  tiled EXT_TILE_TREE_MIXED_RD, spiral N = 10,000,000,
                             r1 = 0.2, r2 = 0.4, 64 x 64 tiles, capacity N + 1
  full_spiral2d_1m_split.npz   tiled, spiral N = 1,000,000, 8 x 8 tiles, capacity
                             50,000 (most tiles are subdivided)
  batch_subset_256.npz       256 clouds of the 4,096-cloud batch (every 16th cloud by
                             size, so the subset spans the whole 1k-200k range, both
                             dims): each cloud's final ridge

All outputs come from oracle/_ref/librdref.so, the reference's CPU code compiled
serially (deterministic) from its own sources by
`make -C oracle ref REF=<checkout>/ridge_detection`.  The batch subset is solved
by a spawn-started process pool, one cloud per task.

Run from the repository root:  python tests/golden/make_golden_fullsize.py [name ...]
"""
from __future__ import annotations

import hashlib
import multiprocessing as mp
import os
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

import oracle as O  # noqa: E402
from ridgedetection_b200 import generators as G  # noqa: E402

OUT = os.path.dirname(os.path.abspath(__file__))


def cloud_sha(P: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(P, np.float32).tobytes()).hexdigest()


def helix_1m():
    n, r1, r2 = 1_000_000, 0.15, 0.3
    P = G.helix3d(n)
    t0 = time.time()
    S_choose = O.ref_choose(P, r1)
    S, passes = S_choose.copy(), []
    for _ in range(5):
        S, _, _, _ = O.ref_evolve_pass(P, S, r1)
        passes.append(S.copy())
    S_final = O.ref_ridge_bf(P, r1, r2)
    np.savez_compressed(os.path.join(OUT, "full_helix3d_1m.npz"), gen="helix3d", n=n,
                        seed=G.SEED_BASE, sha=cloud_sha(P), r1=np.float32(r1),
                        r2=np.float32(r2), S_choose=S_choose, S_passes=np.stack(passes),
                        S_final=S_final)
    print(f"helix 1M: ns_choose={S_choose.shape[0]} ns_final={S_final.shape[0]} "
          f"{time.time() - t0:.0f}s", flush=True)


def tiled(name, n, tpd, cap):
    r1, r2 = 0.2, 0.4
    P = G.spiral2d(n)
    t0 = time.time()
    S, _ = O.ref_ridge_tiled(P, r1, r2, cap, tpd, threads=1)
    np.savez_compressed(os.path.join(OUT, f"{name}.npz"), gen="spiral2d", n=n,
                        seed=G.SEED_BASE, sha=cloud_sha(P), r1=np.float32(r1),
                        r2=np.float32(r2), max_tile_capacity=np.int64(cap),
                        tiles_per_dim=np.array(tpd, np.int64), S_final=S)
    print(f"{name}: ns={S.shape[0]} {time.time() - t0:.0f}s", flush=True)


def batch_subset_ids(spec, count=256):
    """Every (4096 / count)-th cloud in order of size, the largest included."""
    order = sorted(range(len(spec)), key=lambda c: (spec[c][0], c))
    step = len(spec) // count
    ids = [order[len(order) - 1 - k * step] for k in range(count)]
    return sorted(ids)


def _solve_cloud(args):
    c, (n, dim, r1, r2, seed) = args
    P = G.batch_cloud(n, dim, seed)
    return c, O.ref_ridge_bf(P, r1, r2), cloud_sha(P)


def batch_subset():
    spec = G.batch_spec()
    ids = batch_subset_ids(spec)
    t0 = time.time()
    ctx = mp.get_context("spawn")
    with ctx.Pool(max(1, os.cpu_count() or 1)) as pool:
        res = dict((c, (S, sha)) for c, S, sha in
                   pool.imap_unordered(_solve_cloud, [(c, spec[c]) for c in ids]))
    ns = np.array([res[c][0].shape[0] for c in ids], np.int64)
    flat = np.concatenate([res[c][0].reshape(-1) for c in ids]).astype(np.float32)
    np.savez_compressed(os.path.join(OUT, "batch_subset_256.npz"),
                        cloud_ids=np.array(ids, np.int64), ns=ns, S_flat=flat,
                        sha=np.array([res[c][1] for c in ids]))
    sizes = [spec[c][0] for c in ids]
    print(f"batch subset: {len(ids)} clouds, n {min(sizes)}-{max(sizes)}, "
          f"{time.time() - t0:.0f}s", flush=True)


JOBS = {
    "helix": helix_1m,
    "spiral10m": lambda: tiled("full_spiral2d_10m_tiled", 10_000_000, (64, 64), 10_000_001),
    "spiral1m_split": lambda: tiled("full_spiral2d_1m_split", 1_000_000, (8, 8), 50_000),
    "batch": batch_subset,
}


def main(names):
    if O.ref() is None:
        raise SystemExit("oracle/_ref/librdref.so missing: run "
                         "`make -C oracle ref REF=<checkout>/ridge_detection` first")
    for name in names or list(JOBS):
        JOBS[name]()


if __name__ == "__main__":
    main(sys.argv[1:])
