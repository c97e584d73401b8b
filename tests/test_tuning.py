"""Launch-shape tuning table (host side, no GPU needed): buckets, defaults,
argument errors."""
import pytest

import ridgedetection_b200 as rdb


@pytest.fixture(autouse=True)
def _clean():
    rdb.tune_reset()
    yield
    rdb.tune_reset()


def test_default_shape():
    assert rdb.tune_get(2, 20_000) == (128, 8)
    assert rdb.tune_get(3, 1_000_000) == (128, 8)


def test_set_is_per_dim_and_power_of_two_bucket():
    rdb.tune_set(3, 1_000_000, 256, 4)
    assert rdb.tune_get(3, 1_000_000) == (256, 4)
    assert rdb.tune_get(3, 524_288) == (256, 4)     # same bucket [2^19, 2^20)
    assert rdb.tune_get(3, 1_048_576) == (128, 8)   # next bucket
    assert rdb.tune_get(2, 1_000_000) == (128, 8)   # other dim
    rdb.tune_reset()
    assert rdb.tune_get(3, 1_000_000) == (128, 8)


@pytest.mark.parametrize("shape", [(64, 8), (128, 3), (256, 16), (512, 4)])
def test_unsupported_shapes_rejected(shape):
    with pytest.raises(rdb.RDError):
        rdb.tune_set(3, 1000, *shape)


def test_bad_dim_and_size_rejected():
    with pytest.raises(rdb.RDError):
        rdb.tune_set(4, 1000, 128, 8)
    with pytest.raises(rdb.RDError):
        rdb.tune_set(2, 0, 128, 8)
    with pytest.raises(rdb.RDError):
        rdb.tune_get(5, 1000)


def test_assign_cull_switch_roundtrip():
    """The culling switch is process-wide host state: no GPU needed."""
    import ridgedetection_b200 as rdb
    assert rdb.get_assign_cull()
    try:
        rdb.set_assign_cull(False)
        assert not rdb.get_assign_cull()
    finally:
        rdb.set_assign_cull(True)
    assert rdb.get_assign_cull()
