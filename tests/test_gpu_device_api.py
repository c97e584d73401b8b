"""Device-level steps (rd_choose / rd_evolve / rd_decimate) on caller-owned
device buffers vs the reference's outputs (bit-exact)."""
import ctypes
import glob
import os

import numpy as np
import pytest

from gpu_util import bits_equal, require_cuda

pytestmark = pytest.mark.gpu

GOLD = os.path.join(os.path.dirname(__file__), "golden")
BF = sorted(glob.glob(os.path.join(GOLD, "bf_*.npz")))


@pytest.fixture(scope="module")
def env():
    torch = require_cuda()
    from ridgedetection_b200 import _lib as L
    return torch, L


def vp(t):
    return ctypes.c_void_p(t.data_ptr())


@pytest.mark.parametrize("path", BF, ids=[os.path.basename(p)[:-4] for p in BF])
def test_device_steps_match_reference(env, path):
    torch, L = env
    lib = L.lib()
    g = np.load(path)
    P, r1, r2 = g["P"], float(g["r1"]), float(g["r2"])
    n, dim = P.shape
    st = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    dP = torch.from_numpy(P).cuda()
    dS = torch.zeros((max(n, 1), dim), dtype=torch.float32, device="cuda")
    ns = ctypes.c_int64(0)
    L.check(lib.rd_choose(dim, vp(dP), n, r1, vp(dS), ctypes.byref(ns), st))
    assert bits_equal(dS[: ns.value].cpu().numpy(), g["S_choose"])
    passes = ctypes.c_int64(0)
    L.check(lib.rd_evolve(dim, vp(dP), n, vp(dS), ns.value, r1, ctypes.byref(passes), st))
    assert passes.value >= 1
    assert bits_equal(dS[: ns.value].cpu().numpy(), g["S_evolved"])
    left = ctypes.c_int64(0)
    L.check(lib.rd_decimate(dim, vp(dS), ns.value, r2, ctypes.byref(left), st))
    assert bits_equal(dS[: left.value].cpu().numpy(), g["S_decimated"])
