"""Autotuner on the GPU: it picks a supported shape, repeated runs agree
(median of five runs, the incumbent kept within 3%), and every shape gives
bit-identical ridges (shapes change speed only)."""
import pytest

from gpu_util import bits_equal, require_cuda
from ridgedetection_b200 import generators as G

pytestmark = pytest.mark.gpu

CHUNK_SHAPES = [(128, 4), (128, 8), (128, 16), (256, 4), (256, 8)]


@pytest.fixture(scope="module")
def rdb():
    require_cuda()
    import ridgedetection_b200 as rdb
    yield rdb
    rdb.tune_reset()
    rdb.set_assign_cull(True)


@pytest.mark.parametrize("cull", [True, False])
def test_autotune_picks_supported_shape(rdb, cull):
    rdb.tune_reset()
    rdb.set_assign_cull(cull)
    try:
        b, i, ci, us = rdb.autotune(3, 50_000, 200, reps=2, r1=0.1)
    finally:
        rdb.set_assign_cull(True)
    assert (b, i) in CHUNK_SHAPES and ci in (2, 4, 8)
    assert us > 0
    assert rdb.tune_get(3, 50_000, 0.1) == (b, i, ci)


def test_autotune_is_stable_on_the_helix(rdb):
    """Two tunings of the benchmark cloud in a row pick the same shape: the
    second keeps the first unless it loses by more than 3%."""
    torch = require_cuda()
    P = torch.from_numpy(G.helix3d(1_000_000)).cuda()
    rdb.tune_reset()
    first = rdb.autotune(3, 1_000_000, 772, reps=6, points=P, r1=0.15)[:3]
    second = rdb.autotune(3, 1_000_000, 772, reps=6, points=P, r1=0.15)[:3]
    assert first == second
    assert rdb.tune_get(3, 1_000_000, 0.15) == first


@pytest.mark.parametrize("dim", [2, 3])
def test_every_shape_same_ridge(rdb, dim):
    P = G.sine2d(20_000, seed=5) if dim == 2 else G.helix3d(60_000, seed=6)
    r1, r2 = (0.3, 0.6) if dim == 2 else (0.15, 0.3)
    ref = None
    for shape in CHUNK_SHAPES:
        for ci in (2, 4, 8):
            rdb.tune_set(dim, P.shape[0], *shape, ci)
            S, st = rdb.ridge_detection(P, r1, r2)
            assert st.err_bits == 0
            if ref is None:
                ref = S
            else:
                assert bits_equal(S, ref), (shape, ci)
    rdb.tune_reset()


def test_autotune_solve_picks_and_stores_a_shape(rdb):
    """Whole-solve tuning: a supported shape, stored for the bucket, and a
    plausible time per solve; the ridge is the same with the pick."""
    torch = require_cuda()
    P = G.helix3d(60_000, seed=9)
    dP = torch.from_numpy(P).cuda()
    rdb.tune_reset()
    S_before, _ = rdb.ridge_detection(P, 0.15, 0.3)
    b, i, ci, ms = rdb.autotune_solve(3, dP, 0.15, 0.3, runs=1)
    assert (b, i) in CHUNK_SHAPES and ci in (2, 4, 8)
    assert 0.0 < ms < 10_000.0
    assert rdb.tune_get(3, 60_000, 0.15) == (b, i, ci)
    S_after, st = rdb.ridge_detection(P, 0.15, 0.3)
    assert st.err_bits == 0 and bits_equal(S_after, S_before)
    rdb.tune_reset()
