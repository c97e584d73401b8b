"""Chains of a ridge on the GPU (rd_order_chains) == rd::orderSamples
(rd/cpu/brute_force/order.hpp:45) through the oracle, index for index."""
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


def _cases():
    r = np.random.default_rng(2)
    S1, _ = O.ridge_bf(G.sine2d(20000, seed=3), 0.3, 0.6)
    S2, _ = O.ridge_bf(G.helix3d(30000, seed=4), 0.15, 0.3)
    S3 = O.ridge_tiled(G.spiral2d(200000, seed=5), 0.2, 0.4, 200001, (32, 32))[0]
    return [("sine_ridge", S1, 0.6), ("helix_ridge", S2, 0.3), ("spiral_tiled_ridge", S3, 0.4),
            ("random_2d", r.random((5000, 2)).astype(np.float32), 0.03),
            ("random_3d", r.random((3000, 3)).astype(np.float32), 0.08),
            ("line_reversed", np.stack([np.arange(2000)[::-1] * 0.01,
                                        np.zeros(2000)], 1).astype(np.float32), 0.011),
            ("duplicates", np.repeat(r.random((50, 3)).astype(np.float32), 4, axis=0), 0.05),
            ("one", np.zeros((1, 2), np.float32), 0.1),
            ("empty", np.zeros((0, 3), np.float32), 0.1)]


CASES = _cases()


@pytest.mark.parametrize("case", CASES, ids=[c[0] for c in CASES])
def test_order_chains_match_reference(rdb, case):
    _, S, r2 = case
    order, starts = rdb.order_chains(S, r2)
    ref_order, ref_starts = O.ref_order(S, r2) if O.ref(False) is not None else O.order(S, r2)
    assert np.array_equal(starts, ref_starts)
    assert np.array_equal(order, ref_order)


def test_order_of_gpu_ridge(rdb):
    """The device ridge ordered on the device, as a caller would chain it."""
    P = G.helix3d(200_000, seed=9)
    S, st = rdb.ridge_detection(P, 0.15, 0.3)
    order, starts = rdb.order_chains(S, 0.3)
    assert np.array_equal(order, O.order(S, 0.3)[0])
    assert starts[-1] == S.shape[0]
