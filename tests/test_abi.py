"""The C-ABI library loads and exports exactly what include/*.h declares.

CPU-only: no call here reaches the GPU (only argument checks that return
before any CUDA call).
"""
import ctypes
import glob
import os
import re

import pytest

from ridgedetection_b200 import _lib as L

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        src = open(h).read()
        names |= set(re.findall(r"RD_API\s+[\w\s\*]+?\b(rd_\w+)\s*\(", src))
    return names


def test_library_exists_and_loads():
    assert os.path.exists(L.LIB_PATH), "librd_b200.so not built"
    L.lib()


def test_every_declared_symbol_is_exported():
    decl = declared_symbols()
    assert len(decl) >= 18
    raw = ctypes.CDLL(L.LIB_PATH)
    missing = [n for n in sorted(decl) if not hasattr(raw, n)]
    assert not missing, f"declared but not exported: {missing}"


def test_python_binding_covers_header():
    assert declared_symbols() == set(L.SIGNATURES)


def test_argument_errors_need_no_gpu():
    lib = L.lib()
    h = ctypes.c_void_p()
    assert lib.rd_bf_create(None, 2, 0, 0, 10, 0.3, 0.6) == L.RD_ERR_ARG
    assert lib.rd_bf_create(ctypes.byref(h), 7, 0, 0, 10, 0.3, 0.6) == L.RD_ERR_UNSUPPORTED
    assert b"dim" in lib.rd_last_error()
    assert lib.rd_bf_create(ctypes.byref(h), 2, 5, 0, 10, 0.3, 0.6) == L.RD_ERR_ARG
    assert lib.rd_bf_create(ctypes.byref(h), 2, 0, 0, 10, -1.0, 0.6) == L.RD_ERR_ARG
    assert lib.rd_bf_create(ctypes.byref(h), 2, 0, 0, -5, 0.3, 0.6) == L.RD_ERR_ARG
    assert lib.rd_bf_run(None, None) == L.RD_ERR_ARG
    assert lib.rd_batch_run(None, None, 0, None, 0, 0, None) == L.RD_ERR_ARG
    assert lib.rd_abi_version() == 3
    assert lib.rd_supported_dims() & (1 << 2) and lib.rd_supported_dims() & (1 << 3)


def test_cpp_facade_compiles_and_links(tmp_path):
    """include/rd_b200.hpp (the reference-shaped C++ classes) builds against
    librd_b200.so; nothing is run."""
    import shutil
    import subprocess
    cxx = shutil.which("g++")
    if cxx is None:
        pytest.skip("no g++")
    out = tmp_path / "facade"
    cmd = [cxx, "-std=c++14", "-I" + os.path.join(ROOT, "include"), "-I/usr/local/cuda/include",
           os.path.join(ROOT, "tests", "cpp", "facade_compile.cpp"),
           "-L" + os.path.dirname(L.LIB_PATH), "-lrd_b200", "-L/usr/local/cuda/lib64", "-lcudart",
           "-o", str(out)]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-2000:]
