"""The C++ facade (include/rd_b200.hpp) run end to end on a B200: a small
C++ program drives the brute-force and tiled classes the way the reference's
tests drive rd::gpu::bruteForce::RidgeDetection and rd::gpu::tiled::
RidgeDetection, and its ridges are compared bit for bit with the goldens made
by the reference's serial CPU code."""
import os
import shutil
import subprocess

import numpy as np
import pytest

from ridgedetection_b200 import _lib as L

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLD = os.path.join(ROOT, "tests", "golden")

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def facade_bin(tmp_path_factory):
    cxx = shutil.which("g++")
    if cxx is None:
        pytest.skip("no g++")
    out = tmp_path_factory.mktemp("facade") / "facade_run"
    libdir = os.path.dirname(L.LIB_PATH)
    cmd = [cxx, "-std=c++14", "-O1", "-I" + os.path.join(ROOT, "include"), "-I/usr/local/cuda/include",
           os.path.join(ROOT, "tests", "cpp", "facade_run.cpp"), "-L" + libdir, "-lrd_b200",
           "-Wl,-rpath," + libdir, "-L/usr/local/cuda/lib64", "-lcudart", "-o", str(out)]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-2000:]
    return str(out)


def _run(binary, tmp_path, mode, P, r1, r2, extra=()):
    src = tmp_path / "in.bin"
    dst = tmp_path / "out.bin"
    np.ascontiguousarray(P, np.float32).tofile(src)
    cmd = [binary, mode, str(P.shape[1]), str(P.shape[0]), repr(float(r1)), repr(float(r2)),
           str(src), str(dst)] + [str(x) for x in extra]
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, (r.returncode, r.stderr[-2000:])
    raw = dst.read_bytes()
    ns = int(np.frombuffer(raw[:8], np.int64)[0])
    return np.frombuffer(raw[8:], np.float32).reshape(ns, P.shape[1])


def _bits_equal(a, b):
    return a.shape == b.shape and np.array_equal(a.view(np.uint32), b.view(np.uint32))


@pytest.mark.parametrize("name", ["bf_sine2d_3k", "bf_helix3d_5k"])
@pytest.mark.parametrize("mode", ["bf_row", "bf_col"])
def test_facade_brute_force_matches_golden(facade_bin, tmp_path, name, mode):
    g = np.load(os.path.join(GOLD, name + ".npz"))
    # r1 and r2 go through the command line as decimal text; repr() of the
    # float32 value round-trips exactly
    S = _run(facade_bin, tmp_path, mode, g["P"], np.float32(g["r1"]), np.float32(g["r2"]))
    assert _bits_equal(S, g["S_final"])


@pytest.mark.parametrize("mode", ["tiled", "tiled_col"])
def test_facade_tiled_matches_golden(facade_bin, tmp_path, mode):
    g = np.load(os.path.join(GOLD, "tiled_sine2d_5k_tiled.npz"))
    extra = [int(g["max_tile_capacity"])] + [int(t) for t in g["tiles_per_dim"]]
    S = _run(facade_bin, tmp_path, mode, g["P"], np.float32(g["r1"]), np.float32(g["r2"]), extra)
    assert _bits_equal(S, g["S_final"])
