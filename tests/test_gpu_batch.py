"""Batched GPU path: every cloud bit-exact against the CPU restatement."""
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
    return rdb


def small_batch(n_clouds=24, n_min=300, n_max=6000):
    spec = G.batch_spec(n_clouds, seed_base=77, n_min=n_min, n_max=n_max)
    clouds = [(G.batch_cloud(n, dim, seed), r1, r2) for (n, dim, r1, r2, seed) in spec]
    # ragged extremes: a 1-point cloud, a 2-point cloud and an empty cloud
    clouds.append((np.array([[0.1, 0.2]], np.float32), 0.3, 0.6))
    clouds.append((np.array([[0.0, 0.0, 0.0], [0.05, 0.0, 0.0]], np.float32), 0.2, 0.4))
    clouds.append((np.zeros((0, 2), np.float32), 0.3, 0.6))
    return clouds


@pytest.mark.parametrize("mode", ["graph", "host"])
def test_batch_matches_oracle(rdb, mode):
    clouds = small_batch()
    packed, descs = rdb.pack_clouds(clouds)
    b = rdb.BatchedRidgeDetection(rdb.LOOP_GRAPH if mode == "graph" else rdb.LOOP_HOST)
    counts = b.run(packed, descs)
    for c, (P, r1, r2) in enumerate(clouds):
        if P.shape[0] == 0:
            assert counts[c] == 0
            continue
        S_ref, _ = O.ridge_bf(P, r1, r2)
        assert counts[c] == S_ref.shape[0], c
        assert bits_equal(b.chosen_points(c), S_ref), c
    assert b.stats().err_bits == 0
    b.close()


def test_batch_equals_single_cloud_runs(rdb):
    clouds = small_batch(8)[:8]
    packed, descs = rdb.pack_clouds(clouds)
    b = rdb.BatchedRidgeDetection()
    b.run(packed, descs)
    for c, (P, r1, r2) in enumerate(clouds):
        S, _ = rdb.ridge_detection(P, r1, r2)
        assert bits_equal(b.chosen_points(c), S)
    b.close()
