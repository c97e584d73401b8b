"""The acceptance tolerances stated for this path, checked explicitly (the
parity tests already demand bit equality with the reference, which is
stronger):
* evolved positions of every iteration within 1e-5 relative of an FP64
  evaluation of the same assignment (rd/cpu/brute_force/evolve.hpp:43-76 and
  :143-178 restated in double);
* final ridge with the reference's point count and a Hausdorff distance
  <= 1e-4 * r1 (symmetric max-min, assessment_quality.hpp:91-111)."""
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
    from ridgedetection_b200 import autograd
    return rdb, autograd


def test_iterates_within_1e5_of_fp64_same_assignment(rdb):
    _, adj = rdb
    P = G.helix3d(262_144, seed=11)
    r1 = 0.15
    S0 = O.choose(P, r1)
    W = np.zeros(S0.shape, np.float64)
    P64 = P.astype(np.float64)
    prev = S0
    for k in range(1, 6):
        Sk = adj.evolve_adjoint(P, S0, r1, k, W)[0]
        keys = O.assign(P, prev, r1)          # the FP32 assignment of iteration k
        cnt = np.bincount(keys[keys >= 0], minlength=S0.shape[0])
        s64 = np.zeros((S0.shape[0], 3))
        np.add.at(s64, keys[keys >= 0], P64[keys >= 0])
        m = cnt > 0
        mean64 = s64[m] / cnt[m, None]
        rel = np.linalg.norm(Sk[m] - mean64, axis=1) / np.linalg.norm(mean64, axis=1)
        assert rel.max() <= 1e-5, (k, rel.max())
        assert np.array_equal(Sk[~m], prev[~m])  # empty clusters keep their centre
        prev = Sk


@pytest.mark.parametrize("case", ["bf_sine", "bf_helix", "tiled_spiral"])
def test_ridge_count_and_hausdorff(rdb, case):
    api, _ = rdb
    if case == "bf_sine":
        P, r1, r2 = G.sine2d(20_000, seed=21), 0.3, 0.6
        S, st = api.ridge_detection(P, r1, r2)
        S_ref, _ = O.ridge_bf(P, r1, r2)
    elif case == "bf_helix":
        P, r1, r2 = G.helix3d(40_000, seed=22), 0.15, 0.3
        S, st = api.ridge_detection(P, r1, r2)
        S_ref, _ = O.ridge_bf(P, r1, r2)
    else:
        P, r1, r2 = G.spiral2d(200_000, seed=23), 0.2, 0.4
        S, st, _ = api.tiled_ridge_detection(P, r1, r2, P.shape[0] + 1, (32, 32))
        S_ref, _, _ = O.ridge_tiled(P, r1, r2, P.shape[0] + 1, (32, 32))
    assert st.err_bits == 0
    assert S.shape == S_ref.shape
    assert O.hausdorff(S, S_ref) <= 1e-4 * r1
