"""Quality metrics of a ridge on the device (rd_hausdorff, rd_distance_stats,
rd_segment_hausdorff) == the float restatement of
rd/utils/assessment_quality.hpp, which tests/test_oracle.py pins to the
reference's own RDAssessmentQuality<float>."""
import numpy as np
import pytest

import oracle as O
from gpu_util import require_cuda
from ridgedetection_b200 import generators as G

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def rdb():
    require_cuda()
    import ridgedetection_b200 as rdb
    return rdb


def _sets():
    r = np.random.default_rng(8)
    S_sp = O.ridge_tiled(G.spiral2d(100_000, seed=6), 0.2, 0.4, 100_001, (16, 16))[0]
    S_hx, _ = O.ridge_bf(G.helix3d(30_000, seed=7), 0.15, 0.3)
    return [("spiral_ridge", S_sp, G.ideal_spiral2d(50_000, seed=1)),
            ("helix_ridge", S_hx, G.ideal_helix3d(40_000, seed=2)),
            ("random_3d", r.normal(size=(5000, 3)).astype(np.float32),
             r.normal(size=(7000, 3)).astype(np.float32)),
            ("single", np.ones((1, 2), np.float32), np.zeros((3, 2), np.float32)),
            ("odd_sizes", r.random((1025, 2)).astype(np.float32), r.random((1023, 2)).astype(np.float32))]


SETS = _sets()


@pytest.mark.parametrize("case", SETS, ids=[c[0] for c in SETS])
def test_quality_metrics_match_oracle(rdb, case):
    _, T, I = case
    assert np.float32(rdb.hausdorff(T, I)) == np.float32(O.quality(T, I, "hausdorff"))
    got = np.array(rdb.distance_stats(T, I), np.float32)
    want = np.array(O.quality(T, I, "stats"), np.float32)
    assert np.array_equal(got.view(np.uint32), want.view(np.uint32)), (got, want)
    assert np.float32(rdb.segment_hausdorff(T)) == np.float32(O.quality(T, None, "segment"))


def test_empty_test_set(rdb):
    I = np.zeros((4, 2), np.float32)
    assert rdb.hausdorff(np.zeros((0, 2), np.float32), I) == -1.0
    assert rdb.segment_hausdorff(np.zeros((0, 3), np.float32)) == -1.0


def test_quality_of_gpu_ridge_equals_reference_quality(rdb):
    """End to end: ridge and its quality both on the device equal the oracle's
    ridge and quality (the 5% clutter keeps some ridge points off the curve, so
    the distances themselves are not small)."""
    P = G.spiral2d(200_000, seed=10)
    ideal = G.ideal_spiral2d(100_000, seed=3)
    S, st, _ = rdb.tiled_ridge_detection(P, 0.2, 0.4, P.shape[0] + 1, (32, 32))
    S_ref = O.ridge_tiled(P, 0.2, 0.4, P.shape[0] + 1, (32, 32))[0]
    got = np.array(rdb.distance_stats(S, ideal), np.float32)
    want = np.array(O.quality(S_ref, ideal, "stats"), np.float32)
    assert np.array_equal(got, want)
    assert np.float32(rdb.hausdorff(S, ideal)) == np.float32(O.quality(S_ref, ideal, "hausdorff"))
