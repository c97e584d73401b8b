"""Launch-shape tuning table (host side, no GPU needed): buckets by dimension,
size and radius, defaults, argument errors."""
import pytest

import ridgedetection_b200 as rdb


@pytest.fixture(autouse=True)
def _clean():
    rdb.tune_reset()
    yield
    rdb.tune_reset()


def test_default_shape():
    assert rdb.tune_get(2, 20_000, 0.3) == (128, 8, 4)
    assert rdb.tune_get(3, 1_000_000) == (128, 8, 4)


def test_set_is_per_dim_and_power_of_two_bucket():
    rdb.tune_set(3, 1_000_000, 256, 4, 8)
    assert rdb.tune_get(3, 1_000_000) == (256, 4, 8)
    assert rdb.tune_get(3, 524_288) == (256, 4, 8)       # same bucket [2^19, 2^20)
    assert rdb.tune_get(3, 1_048_576) == (128, 8, 4)     # next bucket
    assert rdb.tune_get(2, 1_000_000) == (128, 8, 4)     # other dim
    rdb.tune_reset()
    assert rdb.tune_get(3, 1_000_000) == (128, 8, 4)


def test_radius_buckets():
    """r1 buckets are half octaves; an exact bucket wins over the any-radius
    entry, which wins over the nearest bucket."""
    rdb.tune_set(3, 1_000_000, 256, 8, 2, r1=0.15)
    assert rdb.tune_get(3, 1_000_000, 0.15) == (256, 8, 2)
    assert rdb.tune_get(3, 1_000_000, 0.16) == (256, 8, 2)   # same half octave
    assert rdb.tune_get(3, 1_000_000, 0.6) == (256, 8, 2)    # nearest tuned bucket
    rdb.tune_set(3, 1_000_000, 128, 16, 8, r1=0.6)
    assert rdb.tune_get(3, 1_000_000, 0.6) == (128, 16, 8)
    assert rdb.tune_get(3, 1_000_000, 0.5) == (128, 16, 8)   # nearer to 0.6 than to 0.15
    assert rdb.tune_get(3, 1_000_000, 0.15) == (256, 8, 2)
    rdb.tune_set(3, 1_000_000, 256, 4, 4)                    # any radius
    assert rdb.tune_get(3, 1_000_000, 2.0) == (256, 4, 4)
    assert rdb.tune_get(3, 1_000_000, 0.15) == (256, 8, 2)


@pytest.mark.parametrize("shape", [(64, 8, 4), (128, 3, 4), (256, 16, 4), (512, 4, 4),
                                   (128, 8, 3), (128, 8, 16)])
def test_unsupported_shapes_rejected(shape):
    with pytest.raises(rdb.RDError):
        rdb.tune_set(3, 1000, *shape)


def test_bad_dim_and_size_rejected():
    with pytest.raises(rdb.RDError):
        rdb.tune_set(7, 1000, 128, 8)
    with pytest.raises(rdb.RDError):
        rdb.tune_set(2, 0, 128, 8)
    with pytest.raises(rdb.RDError):
        rdb.tune_get(5, 1000)


def test_assign_cull_switch_roundtrip():
    """The culling switch is process-wide host state: no GPU needed."""
    assert rdb.get_assign_cull()
    try:
        rdb.set_assign_cull(False)
        assert not rdb.get_assign_cull()
    finally:
        rdb.set_assign_cull(True)
    assert rdb.get_assign_cull()


def test_tile_cluster_switch_roundtrip():
    assert rdb.get_tile_clusters() == (True, 100000, 8192)
    try:
        rdb.set_tile_clusters(False, 1000, 64)
        assert rdb.get_tile_clusters() == (False, 1000, 64)
    finally:
        rdb.set_tile_clusters(True, 0, 0)
    assert rdb.get_tile_clusters() == (True, 100000, 8192)
