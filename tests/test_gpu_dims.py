"""Point dimensions other than 2 and 3 (1 and 4): the reference's CPU API
takes the dimension at run time (rd/cpu/brute_force/ridge_detection.hpp:91)
and its GPU classes as a template argument.  Every result here is compared
bit for bit with the reference's own serial CPU code (oracle/_ref) or, for
the tiled variant, with the oracle restatement pinned to it."""
import ctypes

import numpy as np
import pytest

import oracle as O
from gpu_util import bits_equal, require_cuda

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def rdb():
    require_cuda()
    import ridgedetection_b200 as rdb
    return rdb


def line1d(n, seed):
    """Points on a line with gaps: clusters of uneven density."""
    r = np.random.default_rng(seed)
    t = np.concatenate([r.normal(c, s, n // 4) for c, s in ((0, .3), (3, .6), (7, .2), (9, 1.))])
    return np.ascontiguousarray(r.permutation(t)[:, None], dtype=np.float32)


def helix4d(n, seed):
    r = np.random.default_rng(seed)
    t = r.uniform(0, 6 * np.pi, n)
    p = np.stack([np.cos(t), np.sin(t), 0.15 * t, 0.3 * np.sin(2 * t)], 1)
    return np.ascontiguousarray(p + r.normal(0, 0.05, p.shape), dtype=np.float32)


CASES = [("line1d", line1d, 4000, 0.1, 0.2), ("line1d_wide", line1d, 6000, 0.4, 0.8),
         ("helix4d", helix4d, 6000, 0.2, 0.4), ("helix4d_small_r", helix4d, 3000, 0.1, 0.2)]


@pytest.mark.parametrize("name,gen,n,r1,r2", CASES, ids=[c[0] for c in CASES])
def test_brute_force_matches_reference(rdb, name, gen, n, r1, r2):
    P = gen(n, seed=n)
    S_ref = O.ref_ridge_bf(P, r1, r2)
    for lm in (rdb.LOOP_GRAPH, rdb.LOOP_HOST):
        S, st = rdb.ridge_detection(P, r1, r2, loop_mode=lm)
        assert st.err_bits == 0
        assert bits_equal(S, S_ref), (name, S.shape, S_ref.shape)


@pytest.mark.parametrize("name,gen,n,r1,r2,tpd,cap", [
    ("line1d", line1d, 20_000, 0.1, 0.2, (16,), 20_001),
    ("line1d_split", line1d, 20_000, 0.1, 0.2, (4,), 800),
    ("helix4d", helix4d, 20_000, 0.2, 0.4, (2, 2, 3, 1), 20_001),
    ("helix4d_split", helix4d, 20_000, 0.2, 0.4, (2, 1, 2, 1), 1500),
])
def test_tiled_matches_oracle(rdb, name, gen, n, r1, r2, tpd, cap):
    P = gen(n, seed=7)
    S_ref, _, nl_ref = O.ridge_tiled(P, r1, r2, cap, tpd)
    S, st, nl = rdb.tiled_ridge_detection(P, r1, r2, cap, tpd)
    assert st.err_bits == 0 and nl == nl_ref
    assert bits_equal(S, S_ref)


def test_batch_of_mixed_dimensions(rdb):
    clouds = [(line1d(3000, 1), 0.1, 0.2), (helix4d(2500, 2), 0.2, 0.4),
              (line1d(1200, 3), 0.3, 0.6), (helix4d(4000, 4), 0.15, 0.3)]
    packed, descs = rdb.pack_clouds(clouds)
    b = rdb.BatchedRidgeDetection()
    counts = b.run(packed, descs)
    for c, (P, r1, r2) in enumerate(clouds):
        S_ref = O.ref_ridge_bf(P, r1, r2)
        assert counts[c] == S_ref.shape[0]
        assert bits_equal(b.chosen_points(c), S_ref), c
    b.close()


def test_device_steps_in_4d(rdb):
    torch = require_cuda()
    from ridgedetection_b200 import _lib as L
    lib = L.lib()
    P = helix4d(5000, 11)
    r1, r2 = 0.2, 0.4
    n, dim = P.shape
    vp = lambda t: ctypes.c_void_p(t.data_ptr())  # noqa: E731
    st = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    dP = torch.from_numpy(P).cuda()
    dS = torch.zeros_like(dP)
    ns = ctypes.c_int64(0)
    L.check(lib.rd_choose(dim, vp(dP), n, r1, vp(dS), ctypes.byref(ns), st))
    S0 = O.ref_choose(P, r1)
    assert bits_equal(dS[: ns.value].cpu().numpy(), S0)
    passes = ctypes.c_int64(0)
    L.check(lib.rd_evolve(dim, vp(dP), n, vp(dS), ns.value, r1, ctypes.byref(passes), st))
    Se = O.ref_evolve(P, S0, r1)
    assert bits_equal(dS[: ns.value].cpu().numpy(), Se)
    left = ctypes.c_int64(0)
    L.check(lib.rd_decimate(dim, vp(dS), ns.value, r2, ctypes.byref(left), st))
    assert bits_equal(dS[: left.value].cpu().numpy(), O.ref_decimate(Se, r2))


def test_supported_dims_mask(rdb):
    from ridgedetection_b200 import _lib as L
    assert L.lib().rd_supported_dims() == (1 << 1) | (1 << 2) | (1 << 3) | (1 << 4)
