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


def _ws(torch, nbytes):
    return torch.empty(max(int(nbytes), 1), dtype=torch.uint8, device="cuda")


def _col(torch, A, pitch):
    """A (n x dim) as a COL_MAJOR device array with `pitch` floats per coordinate."""
    n, dim = A.shape
    out = torch.full((dim, pitch), float("nan"), dtype=torch.float32, device="cuda")
    out[:, :n] = torch.from_numpy(np.ascontiguousarray(A.T)).cuda()
    return out


@pytest.mark.parametrize("path", BF, ids=[os.path.basename(p)[:-4] for p in BF])
def test_ws_steps_with_layouts_match_reference(env, path):
    """rd_choose_ws / rd_evolve_ws / rd_decimate_ws with caller scratch of
    exactly the queried size, COL_MAJOR pitched and padded ROW_MAJOR arrays,
    and the evolve split into input + neighbour points."""
    torch, L = env
    lib = L.lib()
    g = np.load(path)
    P, r1, r2 = g["P"], float(g["r1"]), float(g["r2"])
    n, dim = P.shape
    st = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    tb = ctypes.c_size_t(0)
    # choose: COL_MAJOR input with a pitch, ROW_MAJOR output padded to dim + 1
    pc = n + 7
    dPc = _col(torch, P, pc)
    dS = torch.full((max(n, 1), dim + 1), float("nan"), dtype=torch.float32, device="cuda")
    L.check(lib.rd_choose_ws(dim, vp(dPc), n, L.RD_COL_MAJOR, pc, r1, None, L.RD_ROW_MAJOR,
                             dim + 1, None, None, ctypes.byref(tb), st))
    ws = _ws(torch, tb.value)
    ns = ctypes.c_int64(0)
    L.check(lib.rd_choose_ws(dim, vp(dPc), n, L.RD_COL_MAJOR, pc, r1, vp(dS), L.RD_ROW_MAJOR,
                             dim + 1, ctypes.byref(ns), vp(ws), ctypes.byref(tb), st))
    S0 = dS[: ns.value, :dim].cpu().numpy()
    assert bits_equal(S0, g["S_choose"])
    k = ns.value
    # one pass, chosen points COL_MAJOR with a pitch, cloud split in two
    cut = n // 3
    dP1 = torch.from_numpy(P[:cut].copy()).cuda()
    dN = _col(torch, P[cut:], n - cut + 5)
    sp = k + 3
    dSc = _col(torch, S0, sp)
    args = lambda w, tbp, mp, pas, mov: (dim, vp(dP1) if cut else None, cut, L.RD_ROW_MAJOR, 0,  # noqa: E731
                                         vp(dN), n - cut, L.RD_COL_MAJOR, n - cut + 5,
                                         vp(dSc), k, L.RD_COL_MAJOR, sp, r1, mp, pas, mov,
                                         w, tbp, st)
    L.check(lib.rd_evolve_ws(*args(None, ctypes.byref(tb), 1, None, None)))
    ws = _ws(torch, tb.value)
    passes, moved = ctypes.c_int64(0), ctypes.c_int32(-1)
    L.check(lib.rd_evolve_ws(*args(vp(ws), ctypes.byref(tb), 1, ctypes.byref(passes),
                                   ctypes.byref(moved))))
    assert passes.value == 1 and moved.value == int(g["cont_pass1"])
    assert bits_equal(dSc[:, :k].T.cpu().numpy(), g["S_pass1"])
    # the rest of the evolve to convergence: same as evolving from S_choose
    dSc = _col(torch, S0, sp)
    L.check(lib.rd_evolve_ws(*args(None, ctypes.byref(tb), 0, None, None)))
    ws = _ws(torch, tb.value)
    L.check(lib.rd_evolve_ws(*args(vp(ws), ctypes.byref(tb), 0, ctypes.byref(passes),
                                   ctypes.byref(moved))))
    assert moved.value == 0
    Se = dSc[:, :k].T.contiguous()
    assert bits_equal(Se.cpu().numpy(), g["S_evolved"])
    assert torch.isnan(dSc[:, k:]).all()
    # decimate in place, COL_MAJOR pitched
    left = ctypes.c_int64(0)
    L.check(lib.rd_decimate_ws(dim, vp(dSc), k, L.RD_COL_MAJOR, sp, r2, None, None,
                               ctypes.byref(tb), st))
    ws = _ws(torch, tb.value)
    L.check(lib.rd_decimate_ws(dim, vp(dSc), k, L.RD_COL_MAJOR, sp, r2, ctypes.byref(left),
                               vp(ws), ctypes.byref(tb), st))
    assert bits_equal(dSc[:, : left.value].T.cpu().numpy(), g["S_decimated"])


def test_ws_rejects_short_or_misaligned_scratch(env):
    torch, L = env
    lib = L.lib()
    g = np.load(os.path.join(GOLD, "bf_sine2d_20k.npz"))
    P, r1 = g["P"], float(g["r1"])
    n, dim = P.shape
    st = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    dP = torch.from_numpy(P).cuda()
    dS = torch.zeros_like(dP)
    tb = ctypes.c_size_t(0)
    L.check(lib.rd_choose_ws(dim, vp(dP), n, 0, 0, r1, None, 0, 0, None, None, ctypes.byref(tb), st))
    need = tb.value
    assert need > n * dim * 4          # holds at least its own copy of the points
    ws = _ws(torch, need + 512)
    short = ctypes.c_size_t(need // 2)
    ns = ctypes.c_int64(0)
    rc = lib.rd_choose_ws(dim, vp(dP), n, 0, 0, r1, vp(dS), 0, 0, ctypes.byref(ns), vp(ws),
                          ctypes.byref(short), st)
    assert rc == L.RD_ERR_CAPACITY and b"temporary storage" in lib.rd_last_error()
    odd = ctypes.c_void_p(ws.data_ptr() + 16)
    rc = lib.rd_choose_ws(dim, vp(dP), n, 0, 0, r1, vp(dS), 0, 0, ctypes.byref(ns), odd,
                          ctypes.byref(tb), st)
    assert rc == L.RD_ERR_ARG
    # the query does not depend on the data, and a call after a failure works
    L.check(lib.rd_choose_ws(dim, vp(dP), n, 0, 0, r1, vp(dS), 0, 0, ctypes.byref(ns), vp(ws),
                             ctypes.byref(tb), st))
    assert bits_equal(dS[: ns.value].cpu().numpy(), g["S_choose"])


def test_evolve_pass_entry_point(env):
    torch, L = env
    lib = L.lib()
    g = np.load(os.path.join(GOLD, "bf_helix3d_20k.npz"))
    P, r1 = g["P"], float(g["r1"])
    st = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    dP = torch.from_numpy(P).cuda()
    dS = torch.from_numpy(g["S_choose"]).cuda()
    moved = ctypes.c_int32(-1)
    L.check(lib.rd_evolve_pass(3, vp(dP), P.shape[0], vp(dS), dS.shape[0], r1,
                               ctypes.byref(moved), st))
    assert moved.value == int(g["cont_pass1"])
    assert bits_equal(dS.cpu().numpy(), g["S_pass1"])
