"""Brute-force GPU path vs the reference's outputs and the CPU restatement.

Bit-exact: the final chosen points (count, order and every float bit) must
equal the reference's serial CPU result on the same input.
"""
import glob
import os

import numpy as np
import pytest

import oracle as O
from gpu_util import bits_equal, decimation_is_stable, require_cuda
from ridgedetection_b200 import generators as G

pytestmark = pytest.mark.gpu

GOLD = os.path.join(os.path.dirname(__file__), "golden")
BF = sorted(glob.glob(os.path.join(GOLD, "bf_*.npz")))


@pytest.fixture(scope="module")
def rdb():
    require_cuda()
    import ridgedetection_b200 as rdb
    return rdb


@pytest.mark.parametrize("mode", ["graph", "host"])
@pytest.mark.parametrize("path", BF, ids=[os.path.basename(p)[:-4] for p in BF])
def test_bf_matches_reference_golden(rdb, path, mode):
    g = np.load(path)
    lm = rdb.LOOP_GRAPH if mode == "graph" else rdb.LOOP_HOST
    S, st = rdb.ridge_detection(g["P"], float(g["r1"]), float(g["r2"]), loop_mode=lm)
    assert bits_equal(S, g["S_final"]), (S.shape, g["S_final"].shape)
    assert st.err_bits == 0


@pytest.mark.parametrize("seed", [1, 2, 3])
@pytest.mark.parametrize("kind", ["sine", "helix"])
def test_bf_matches_oracle_seeded(rdb, kind, seed):
    if kind == "sine":
        P, r1, r2 = G.sine2d(4000 + 1500 * seed, seed=100 + seed), 0.25 + 0.02 * seed, 0.5 + 0.04 * seed
    else:
        P, r1, r2 = G.helix3d(3000 + 2000 * seed, seed=200 + seed), 0.12 + 0.03 * seed, 0.24 + 0.06 * seed
    S_ref, st_ref = O.ridge_bf(P, r1, r2)
    S, st = rdb.ridge_detection(P, r1, r2)
    assert bits_equal(S, S_ref)
    assert st.evolve_passes == st_ref.evolve_passes
    assert abs(st.pairs - st_ref.pairs) < 0.5


def test_bf_layouts_and_pitches(rdb):
    g = np.load(os.path.join(GOLD, "bf_helix3d_5k.npz"))
    P, r1, r2, ref = g["P"], float(g["r1"]), float(g["r2"]), g["S_final"]
    n, dim = P.shape
    # COL_MAJOR input with a pitch larger than n, COL_MAJOR output with a pitch
    pitch_in = n + 37
    col = np.zeros((dim, pitch_in), np.float32)
    col[:, :n] = P.T
    rd = rdb.BruteForceRidgeDetection(n, r1, r2, dim, in_layout=rdb.COL_MAJOR,
                                      out_layout=rdb.COL_MAJOR)
    rd.set_points(col, pitch=pitch_in)
    rd.ridge_detection()
    ns = rd.get_chosen_samples_count()
    assert ns == ref.shape[0]
    pitch_out = ns + 5
    out = np.full((dim, pitch_out), np.nan, np.float32)
    rd.chosen_points(out, pitch=pitch_out)
    assert bits_equal(out[:, :ns].T, ref)
    assert np.isnan(out[:, ns:]).all()
    rd.close()
    # ROW_MAJOR input with padding between points
    padded = np.zeros((n, dim + 2), np.float32)
    padded[:, :dim] = P
    rd = rdb.BruteForceRidgeDetection(n, r1, r2, dim)
    rd.set_points(padded, pitch=dim + 2)
    rd.ridge_detection()
    assert bits_equal(rd.chosen_points(), ref)
    rd.close()


def test_bf_device_tensors_and_rerun(rdb):
    torch = require_cuda()
    g = np.load(os.path.join(GOLD, "bf_sine2d_20k.npz"))
    P = torch.from_numpy(g["P"]).cuda()
    rd = rdb.BruteForceRidgeDetection(P.shape[0], float(g["r1"]), float(g["r2"]), 2)
    for _ in range(2):  # the handle is reusable; results must not drift
        rd.set_points(P)
        rd.ridge_detection()
        out = torch.empty((rd.ns_, 2), dtype=torch.float32, device="cuda")
        rd.chosen_points(out)
        torch.cuda.synchronize()
        assert bits_equal(out.cpu().numpy(), g["S_final"])
    rd.close()


def test_bf_full_size_helix_properties(rdb):
    """1M-point helix: deterministic, graph == host loop, and the result is a
    fixed point of both evolve (one more pass moves nothing) and decimate.
    (Bit parity with the reference at this size: tests/test_gpu_fullsize.py.)"""
    P = G.helix3d(1_000_000)
    r1, r2 = 0.15, 0.3
    S1, st1 = rdb.ridge_detection(P, r1, r2, loop_mode=rdb.LOOP_GRAPH)
    S2, st2 = rdb.ridge_detection(P, r1, r2, loop_mode=rdb.LOOP_HOST)
    assert bits_equal(S1, S2)
    assert st1.evolve_passes == st2.evolve_passes and st1.err_bits == 0
    S_after, _, _, _, cont = O.evolve_pass(P, S1, r1)
    assert cont == 0 and bits_equal(S_after, S1)
    assert decimation_is_stable(S1, r2)


@pytest.mark.parametrize("centre", [0.0, -0.5])
def test_bf_big_clusters_cta_fold(rdb, centre):
    """Clusters of more than 16,384 members (folded by whole CTAs with the
    warp-segmented exact fold in k_sum_shift), including coordinate sums that
    wander around zero (centre -0.5: the cube straddles the origin)."""
    P = (np.random.default_rng(77).uniform(0, 1, (300_000, 3)) + centre).astype(np.float32)
    r1, r2 = 0.6, 1.2
    S0 = O.choose(P, np.float32(r1))
    _, _, cnt, _, _ = O.evolve_pass(P, S0, np.float32(r1))
    assert cnt.max() >= 16384  # the CTA path is exercised
    S_ref, _ = O.ridge_bf(P, np.float32(r1), np.float32(r2))
    S, st = rdb.ridge_detection(P, r1, r2)
    assert st.err_bits == 0
    assert bits_equal(S, S_ref)
