"""Ordered FP32 sums (rd_ordered_sum): the add chain, the warp-parallel, the
CTA-wide and the warp-segmented (8 and 32 segments) exact evaluations must all
reproduce the serial loop of rd/cpu/brute_force/evolve.hpp:71-74 bit for bit,
including ties, binade crossings, cancellation and non-finite terms."""
import ctypes

import numpy as np
import pytest

from gpu_util import require_cuda

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def env():
    require_cuda()
    import torch
    from ridgedetection_b200 import _lib as L
    return torch, L


def serial_sum(X, idx):
    """Left-to-right float32 sum from 0 of X[idx, d] (numpy accumulate is serial)."""
    out = []
    for d in range(X.shape[1]):
        seq = np.concatenate([np.zeros(1, np.float32), X[idx, d].astype(np.float32)])
        out.append(np.add.accumulate(seq, dtype=np.float32)[-1])
    return np.array(out, np.float32)


def gpu_sum(env, X, idx, method):
    torch, L = env
    dP = torch.from_numpy(np.ascontiguousarray(X, np.float32)).cuda()
    dI = torch.from_numpy(np.ascontiguousarray(idx, np.int32)).cuda()
    out = torch.zeros(X.shape[1], dtype=torch.float32, device="cuda")
    vp = ctypes.c_void_p
    L.check(L.lib().rd_ordered_sum(X.shape[1], vp(dP.data_ptr()), vp(dI.data_ptr()), len(idx),
                                   vp(out.data_ptr()), method, None))
    return out.cpu().numpy()


def same(a, b):
    a, b = np.asarray(a, np.float32), np.asarray(b, np.float32)
    nan = np.isnan(a) & np.isnan(b)
    return bool(np.all(nan | (a.view(np.uint32) == b.view(np.uint32))))


def _cases():
    r = np.random.default_rng(7)
    cases = {}
    n = 200_000
    cases["normal"] = r.normal(size=(n, 3)).astype(np.float32)
    cases["positive"] = r.random((300_000, 2)).astype(np.float32)
    cases["walk_near_zero"] = r.normal(0, 0.1, size=(n, 2)).astype(np.float32)
    cases["centred_cluster"] = (r.normal(0, 0.05, size=(n, 2)) + np.array([1e-3, -2e-4])).astype(np.float32)
    # multiples of 1/4: once the sum passes 2^22 every term lands on or next to
    # a rounding tie
    cases["ties"] = (r.integers(-32, 256, size=(1_000_000, 2)) * 0.25).astype(np.float32)
    cases["ties_negative"] = (r.integers(-256, 32, size=(1_000_000, 3)) * 0.5).astype(np.float32)
    mag = 10.0 ** r.uniform(-20, 20, size=(n, 2))
    cases["magnitudes"] = (r.normal(size=(n, 2)) * mag).astype(np.float32)
    x = r.normal(size=(50_000, 2)).astype(np.float32)
    cases["cancel"] = np.concatenate([x, -x[::-1], x[:1000]])  # returns to exactly 0 midway
    big = np.full((20_000, 2), 3.0e36, np.float32)
    big[::7] *= -1
    cases["overflow"] = big
    sp = r.normal(size=(40_000, 2)).astype(np.float32)
    sp[::1000, 0] = np.inf
    sp[5::1000, 1] = -0.0
    sp[17::999, 1] = np.float32(1e-45)
    cases["specials"] = sp
    nanc = r.normal(size=(10_000, 2)).astype(np.float32)
    nanc[4321, 1] = np.nan
    cases["nan"] = nanc
    cases["subnormal"] = (r.normal(size=(30_000, 2)) * 1e-40).astype(np.float32)
    return cases


CASES = _cases()


@pytest.mark.parametrize("method", [0, 1, 2, 3, 4])
@pytest.mark.parametrize("name", sorted(CASES))
def test_ordered_sum_matches_serial(env, name, method):
    X = CASES[name]
    r = np.random.default_rng(len(name))
    for idx in (np.arange(X.shape[0]), np.sort(r.choice(X.shape[0], X.shape[0] // 3, replace=False)),
                r.permutation(X.shape[0])):
        got = gpu_sum(env, X, idx, method)
        want = serial_sum(X, idx)
        assert same(got, want), (name, method, got, want)


@pytest.mark.parametrize("n", [0, 1, 2, 7, 31, 32, 33, 255, 256, 257, 511, 2047, 2049, 4097, 70001])
def test_ordered_sum_ragged_sizes(env, n):
    X = np.random.default_rng(n).normal(size=(max(n, 1), 2)).astype(np.float32) + 3.0
    idx = np.arange(n)
    want = serial_sum(X, idx)
    for method in (0, 1, 2, 3, 4):
        assert same(gpu_sum(env, X, idx, method), want), (n, method)


def test_serial_reference_is_a_loop():
    X = np.random.default_rng(1).normal(size=(3000, 2)).astype(np.float32) * 1e3
    idx = np.arange(3000)
    s = [np.float32(0), np.float32(0)]
    for i in idx:
        for d in range(2):
            s[d] = np.float32(s[d] + X[i, d])
    assert same(np.array(s, np.float32), serial_sum(X, idx))
