"""Autotuner on the GPU: it picks a supported shape, and every shape gives
bit-identical ridges (shapes change speed only)."""
import pytest

from gpu_util import bits_equal, require_cuda
from ridgedetection_b200 import generators as G

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def rdb():
    require_cuda()
    import ridgedetection_b200 as rdb
    yield rdb
    rdb.tune_reset()


def test_autotune_picks_supported_shape(rdb):
    b, i, us = rdb.autotune(3, 50_000, 200, reps=2)
    assert (b, i) in {(128, 4), (128, 8), (128, 16), (256, 4), (256, 8)}
    assert us > 0
    assert rdb.tune_get(3, 50_000) == (b, i)


@pytest.mark.parametrize("dim", [2, 3])
def test_every_shape_same_ridge(rdb, dim):
    P = G.sine2d(20_000, seed=5) if dim == 2 else G.helix3d(60_000, seed=6)
    r1, r2 = (0.3, 0.6) if dim == 2 else (0.15, 0.3)
    ref = None
    for shape in [(128, 4), (128, 8), (128, 16), (256, 4), (256, 8)]:
        rdb.tune_set(dim, P.shape[0], *shape)
        S, st = rdb.ridge_detection(P, r1, r2)
        assert st.err_bits == 0
        if ref is None:
            ref = S
        else:
            assert bits_equal(S, ref), shape
    rdb.tune_reset()
