"""Tiled GPU path vs the reference's EXT_TILE_TREE_MIXED_RD outputs (bit-exact)."""
import glob
import os

import numpy as np
import pytest

import oracle as O
from gpu_util import bits_equal, decimation_is_stable, require_cuda
from ridgedetection_b200 import generators as G

pytestmark = pytest.mark.gpu

GOLD = os.path.join(os.path.dirname(__file__), "golden")
TILED = sorted(glob.glob(os.path.join(GOLD, "tiled_*.npz")))


@pytest.fixture(scope="module")
def rdb():
    require_cuda()
    import ridgedetection_b200 as rdb
    return rdb


@pytest.mark.parametrize("mode", ["graph", "host"])
@pytest.mark.parametrize("path", TILED, ids=[os.path.basename(p)[:-4] for p in TILED])
def test_tiled_matches_reference_golden(rdb, path, mode):
    g = np.load(path)
    lm = rdb.LOOP_GRAPH if mode == "graph" else rdb.LOOP_HOST
    S, st, nl = rdb.tiled_ridge_detection(g["P"], float(g["r1"]), float(g["r2"]),
                                          int(g["max_tile_capacity"]), g["tiles_per_dim"],
                                          loop_mode=lm)
    assert bits_equal(S, g["S_final"]), (S.shape, g["S_final"].shape)
    assert st.err_bits == 0


@pytest.mark.parametrize("case", [
    ("spiral", 60_000, 0.2, 0.4, 60_001, (16, 16)),
    ("spiral_split", 30_000, 0.2, 0.4, 1500, (3, 5)),
    ("helix", 40_000, 0.15, 0.3, 40_001, (4, 4, 3)),
    ("sine_one_tile", 5_000, 0.3, 0.6, 5_001, (1, 1)),
    # 3106 tiles: the global decimation holds more than 4096 chosen points
    # (GPU-wide preparation) with neighbour lists long enough for the
    # CTA-wide count updates
    ("spiral_4k_tiles", 200_000, 0.2, 0.4, 200_001, (64, 64)),
])
def test_tiled_matches_oracle(rdb, case):
    kind, n, r1, r2, cap, tpd = case
    P = {"spiral": lambda: G.spiral2d(n, seed=41), "spiral_split": lambda: G.spiral2d(n, seed=42),
         "helix": lambda: G.helix3d(n, seed=43), "sine_one_tile": lambda: G.sine2d(n, seed=44),
         "spiral_4k_tiles": lambda: G.spiral2d(n, seed=45)}[kind]()
    S_ref, st_ref, nl_ref = O.ridge_tiled(P, r1, r2, cap, tpd)
    S, st, nl = rdb.tiled_ridge_detection(P, r1, r2, cap, tpd)
    assert nl == nl_ref
    assert bits_equal(S, S_ref)
    assert st.evolve_passes <= st_ref.evolve_passes  # unchanged tiles may skip nothing here


def test_tiled_spiral_10m_properties(rdb):
    """The benchmark-size tiled cloud (10M points, 64x64 tiles): deterministic,
    graph == host loop, and the final set is stable under another decimation."""
    P = G.spiral2d(10_000_000)
    args = (0.2, 0.4, 10_000_001, (64, 64))
    S1, st1, nl1 = rdb.tiled_ridge_detection(P, *args, loop_mode=rdb.LOOP_GRAPH)
    S2, st2, nl2 = rdb.tiled_ridge_detection(P, *args, loop_mode=rdb.LOOP_HOST)
    assert nl1 == nl2 and bits_equal(S1, S2) and st1.err_bits == 0
    assert S1.shape[0] > 100
    if S1.shape[0] <= 8000:
        assert decimation_is_stable(S1, 0.4)


@pytest.mark.parametrize("case", [
    ("spiral_split", 30_000, 0.2, 0.4, 1500, (3, 5)),
    ("sine_2x2", 20_000, 0.3, 0.6, 20_001, (2, 2)),
    ("helix_2x2x2", 20_000, 0.15, 0.3, 20_001, (2, 2, 2)),
])
def test_tiled_end_phase_refinement_matches_oracle(rdb, case):
    """end_phase_refinement = 1: the tiled result, then a brute-force decimation
    and an evolve of the whole cloud (rd/cpu/tiled/rd_tiled.hpp:1386-1419)."""
    kind, n, r1, r2, cap, tpd = case
    P = {"spiral_split": lambda: G.spiral2d(n, seed=42), "sine_2x2": lambda: G.sine2d(n, seed=46),
         "helix_2x2x2": lambda: G.helix3d(n, seed=47)}[kind]()
    S_ref, _, nl_ref = O.ridge_tiled(P, r1, r2, cap, tpd, refine=True)
    S, st, nl = rdb.tiled_ridge_detection(P, r1, r2, cap, tpd, end_phase_refinement=True)
    assert nl == nl_ref
    assert bits_equal(S, S_ref)


@pytest.mark.parametrize("case", [
    ("spiral", 60_000, 0.2, 0.4, 60_001, (16, 16), False),
    ("spiral_split", 30_000, 0.2, 0.4, 1500, (3, 5), False),
    ("helix", 40_000, 0.15, 0.3, 40_001, (4, 4, 3), False),
    ("spiral_split_refined", 30_000, 0.2, 0.4, 1500, (3, 5), True),
])
def test_tiled_local_policy_matches_oracle(rdb, case):
    """RD_LOCAL: a complete ridge detection inside every leaf (the reference's
    GPU RD_LOCAL policy; no CPU counterpart exists, the oracle restates it)."""
    kind, n, r1, r2, cap, tpd, refine = case
    P = {"spiral": lambda: G.spiral2d(n, seed=41), "spiral_split": lambda: G.spiral2d(n, seed=42),
         "helix": lambda: G.helix3d(n, seed=43),
         "spiral_split_refined": lambda: G.spiral2d(n, seed=42)}[kind]()
    S_ref, _, nl_ref = O.ridge_tiled_local(P, r1, r2, cap, tpd, refine=refine)
    S, st, nl = rdb.tiled_ridge_detection(P, r1, r2, cap, tpd, end_phase_refinement=refine,
                                          policy=rdb.TILED_LOCAL)
    assert nl == nl_ref
    assert st.err_bits == 0
    assert bits_equal(S, S_ref)


@pytest.mark.parametrize("case", [
    # deep subdivision: a small capacity splits tiles over many levels
    ("spiral_deep", 30_000, 0.2, 0.4, 200, (2, 2)),
    ("helix_deep", 30_000, 0.15, 0.3, 300, (2, 1, 2)),
    ("sine_deep", 20_000, 0.3, 0.6, 150, (3, 1)),
])
def test_device_subdivision_matches_oracle(rdb, case):
    """Tiles with max_tile_capacity or more own points are split level by level
    on the device (grouped_tile_tree.inl:247-330); the leaves, their order and
    the ridge equal the oracle's."""
    kind, n, r1, r2, cap, tpd = case
    P = {"spiral_deep": lambda: G.spiral2d(n, seed=51), "helix_deep": lambda: G.helix3d(n, seed=52),
         "sine_deep": lambda: G.sine2d(n, seed=53)}[kind]()
    S_ref, _, nl_ref = O.ridge_tiled(P, r1, r2, cap, tpd)
    S, st, nl = rdb.tiled_ridge_detection(P, r1, r2, cap, tpd)
    assert nl == nl_ref and nl > 20
    assert bits_equal(S, S_ref) and st.err_bits == 0


def test_subdivision_of_duplicates_is_an_error(rdb):
    """Identical points above the capacity can never be separated: the split
    gives up after 64 levels with an error instead of looping."""
    P = np.zeros((500, 2), np.float32)
    P[:250] = 1.0
    with pytest.raises(rdb.RDError):
        rdb.tiled_ridge_detection(P, 0.2, 0.4, 100, (1, 1))
