"""rd_decimate_noalloc: the decimation for callers that cannot allocate device
memory (hosts that forbid device allocation once they have started, plugins
whose framework gives them no workspace).  Its scratch is a fixed array inside
the library; it must give exactly what the allocating rd_decimate gives, call
after call, since every call reuses (and must re-clear) that array.

Collected last on purpose (file name), so a failure here cannot hide the
results of the other tests.
"""
import ctypes
import glob
import os

import numpy as np
import pytest

from gpu_util import bits_equal, require_cuda

pytestmark = pytest.mark.gpu

GOLD = os.path.join(os.path.dirname(__file__), "golden")


def _sets():
    out = []
    for path in sorted(glob.glob(os.path.join(GOLD, "bf_*.npz"))):
        g = np.load(path)
        out.append((os.path.basename(path), g["S_evolved"], float(g["r2"])))
    rng = np.random.default_rng(12)
    # larger sets, near the fixed limit, dense enough that decimation removes many
    t = rng.uniform(0, 60, 30000)
    big3 = np.stack([np.cos(t), np.sin(t), 0.15 * t], 1) + rng.normal(0, 0.05, (30000, 3))
    out.append(("helix_30000", big3.astype(np.float32), 0.3))
    big2 = rng.uniform(-20, 20, (32768, 2)).astype(np.float32)
    out.append(("uniform_32768", big2, 0.5))
    return out


def test_noalloc_matches_allocating_decimate_twice_in_a_row():
    torch = require_cuda()
    from ridgedetection_b200 import _lib as L
    lib = L.lib()
    st = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    for name, S, r2 in _sets():
        ns, dim = S.shape
        ref = torch.from_numpy(S).cuda()
        left = ctypes.c_int64(0)
        L.check(lib.rd_decimate(dim, ctypes.c_void_p(ref.data_ptr()), ns, r2,
                                ctypes.byref(left), st))
        expect = ref[: left.value].cpu().numpy()
        for call in range(2):
            d = torch.from_numpy(S).cuda()
            cnt = torch.full((1,), -7, dtype=torch.int32, device="cuda")
            L.check(lib.rd_decimate_noalloc(dim, ctypes.c_void_p(d.data_ptr()), ns, r2,
                                            ctypes.c_void_p(cnt.data_ptr()), st))
            torch.cuda.synchronize()
            got = int(cnt.item())
            assert got == left.value, (name, call, got, left.value)
            assert bits_equal(d[:got].cpu().numpy(), expect), (name, call)


def test_noalloc_rejects_sizes_beyond_its_limit():
    torch = require_cuda()
    from ridgedetection_b200 import _lib as L
    lib = L.lib()
    n = 32769
    d = torch.zeros((n, 2), dtype=torch.float32, device="cuda")
    cnt = torch.zeros((1,), dtype=torch.int32, device="cuda")
    rc = lib.rd_decimate_noalloc(2, ctypes.c_void_p(d.data_ptr()), n, 0.5,
                                 ctypes.c_void_p(cnt.data_ptr()), ctypes.c_void_p(0))
    assert rc == L.RD_ERR_CAPACITY
    assert b"32768" in lib.rd_last_error()
