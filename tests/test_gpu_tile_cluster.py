"""Cluster evolve of heavy tiles (rd_tile_cluster.cuh) against the oracle and
against one CTA per tile, bit for bit.

The thresholds are lowered so that small clouds send most tiles through the
cluster path and fold most keys in segments: the per-CTA count exchange, the
placement offsets, the speculative segment folds and their composition (runs
on one grid, chunks folded exactly at binade crossings, fallbacks when a trace
does not apply -- sums that wander around zero produce many of those) and the
gathering of every key's result.
"""
import numpy as np
import pytest

import oracle as O
from gpu_util import bits_equal, require_cuda
from ridgedetection_b200 import generators as G

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def rdb():
    require_cuda()
    import ridgedetection_b200 as rdb
    yield rdb
    rdb.set_tile_clusters(True, 0, 0)


def centred_uniform(n, seed):
    """Uniform in [-1, 1]^2: with a large r1 every cluster's coordinate sums
    wander around zero (many binade changes and sign changes)."""
    return np.random.default_rng(seed).uniform(-1, 1, (n, 2)).astype(np.float32)


CASES = {
    # name: (cloud, r1, r2, capacity, tiles per dim)
    "spiral_16x16": (lambda: G.spiral2d(60_000, seed=41), 0.2, 0.4, 60_001, (16, 16)),
    "spiral_split": (lambda: G.spiral2d(30_000, seed=42), 0.2, 0.4, 1500, (3, 5)),
    "helix_3d": (lambda: G.helix3d(40_000, seed=43), 0.15, 0.3, 40_001, (4, 4, 3)),
    "around_zero": (lambda: centred_uniform(40_000, 7), 0.6, 1.2, 40_001, (2, 2)),
    "many_keys": (lambda: centred_uniform(50_000, 8), 0.03, 0.06, 50_001, (2, 2)),
    "spiral_64x64": (lambda: G.spiral2d(200_000, seed=45), 0.2, 0.4, 200_001, (64, 64)),
}


@pytest.mark.parametrize("seg_min", [1, 64, 4096])
@pytest.mark.parametrize("name", list(CASES))
def test_cluster_tiles_match_oracle(rdb, name, seg_min):
    gen, r1, r2, cap, tpd = CASES[name]
    P = gen()
    S_ref, _, nl_ref = O.ridge_tiled(P, r1, r2, cap, tpd)
    rdb.set_tile_clusters(True, 64, seg_min)
    try:
        S, st, nl = rdb.tiled_ridge_detection(P, r1, r2, cap, tpd)
        S_host, _, _ = rdb.tiled_ridge_detection(P, r1, r2, cap, tpd, loop_mode=rdb.LOOP_HOST)
    finally:
        rdb.set_tile_clusters(True, 0, 0)
    assert nl == nl_ref and st.err_bits == 0
    assert bits_equal(S, S_ref), (S.shape, S_ref.shape)
    assert bits_equal(S_host, S_ref)


def test_cluster_switch_changes_nothing(rdb):
    P = G.spiral2d(1_000_000, seed=46)
    args = (0.2, 0.4, 1_000_001, (32, 32))
    rdb.set_tile_clusters(False)
    try:
        S_off, _, _ = rdb.tiled_ridge_detection(P, *args)
    finally:
        rdb.set_tile_clusters(True, 0, 0)
    S_on, st, _ = rdb.tiled_ridge_detection(P, *args)
    assert st.err_bits == 0 and bits_equal(S_on, S_off)
    assert rdb.get_tile_clusters() == (True, 100000, 8192)
