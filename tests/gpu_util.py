"""Helpers shared by the GPU parity tests."""
import numpy as np
import pytest


def bits_equal(a, b):
    a = np.ascontiguousarray(a, np.float32)
    b = np.ascontiguousarray(b, np.float32)
    return a.shape == b.shape and np.array_equal(a.view(np.uint32), b.view(np.uint32))


def require_cuda():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


def decimation_is_stable(S, r2):
    """No point of S would be removed by another decimation pass
    (rd/cpu/brute_force/decimate.hpp:58-66)."""
    S = np.asarray(S, np.float32)
    if S.shape[0] <= 3:
        return True
    r = np.float32(r2)
    rsq = np.float32(r * r)
    rsq4 = np.float32(np.float32(4.0) * rsq)
    acc = np.zeros((S.shape[0], S.shape[0]), np.float32)
    for d in range(S.shape[1]):
        t = (S[:, None, d] - S[None, :, d]).astype(np.float32)
        acc = (acc + (t * t).astype(np.float32)).astype(np.float32)
    c1 = (acc <= rsq).sum(1)
    c2 = (acc <= rsq4).sum(1)
    return not np.any((c1 >= 4) | (c2 < 3))
