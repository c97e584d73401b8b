"""Evolve adjoint on the GPU: forward bit-exact, gradients against the FP64 CPU
reverse pass and against central finite differences (h = 1e-3, FP64)."""
import numpy as np
import pytest

import oracle as O
from gpu_util import bits_equal, require_cuda
from ridgedetection_b200 import generators as G

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def adj():
    require_cuda()
    from ridgedetection_b200 import autograd
    return autograd


def chosen_indices(P, S):
    """Row index of every chosen point (choose copies the first occurrence)."""
    first = {}
    for i, row in enumerate(P.view(np.uint32).reshape(P.shape[0], -1)):
        first.setdefault(row.tobytes(), i)
    return np.array([first[r.tobytes()] for r in S.view(np.uint32).reshape(S.shape[0], -1)])


def assign64(P, S, r1):
    d = ((P[:, None, :] - S[None, :, :]) ** 2).sum(-1)
    k = d.argmin(1)
    k[d[np.arange(P.shape[0]), k] > r1 * r1] = -1
    return k


def forward64(P, S0, r1, iters, keys=None):
    """FP64 forward; with `keys` the assignments are frozen, else recomputed."""
    S = S0.astype(np.float64).copy()
    seq = []
    for t in range(iters):
        k = keys[t] if keys is not None else assign64(P, S, r1)
        seq.append(k)
        m = k >= 0
        cnt = np.bincount(k[m], minlength=S.shape[0])
        out = S.copy()
        nz = cnt > 0
        for d in range(P.shape[1]):
            sums = np.bincount(k[m], weights=P[m, d], minlength=S.shape[0])
            out[nz, d] = sums[nz] / cnt[nz]
        S = out
    return S, seq


@pytest.mark.parametrize("ckpt", [0, 5])
def test_adjoint_matches_fp64_oracle(adj, ckpt):
    P = G.helix3d(4000, seed=31)
    r1 = 0.2
    S0 = O.choose(P, r1)
    W = np.random.default_rng(3).normal(size=S0.shape)
    Sf, gP, gS = adj.evolve_adjoint(P, S0, r1, 12, W, checkpoint_every=ckpt)
    gP_ref, gS_ref, Sf_ref = O.evolve_adjoint(P, S0, r1, 12, W)
    assert bits_equal(Sf, Sf_ref)
    np.testing.assert_allclose(gP, gP_ref, rtol=1e-12, atol=1e-15)
    np.testing.assert_allclose(gS, gS_ref, rtol=1e-12, atol=1e-15)


def test_adjoint_checkpointing_is_exact(adj):
    P = G.sine2d(6000, seed=32)
    r1 = 0.25
    S0 = O.choose(P, r1)
    W = np.random.default_rng(4).normal(size=S0.shape)
    a = adj.evolve_adjoint(P, S0, r1, 20, W, checkpoint_every=0)
    b = adj.evolve_adjoint(P, S0, r1, 20, W, checkpoint_every=5)
    c = adj.evolve_adjoint(P, S0, r1, 20, W, checkpoint_every=7)
    for x, y in ((a, b), (a, c)):
        assert bits_equal(x[0], y[0])
        assert np.array_equal(x[1], y[1]) and np.array_equal(x[2], y[2])


def test_adjoint_true_finite_differences_small(adj):
    """FP64 central differences with the assignment recomputed in FP64, on
    coordinates whose perturbed runs keep every assignment (away from ball and
    Voronoi boundaries): relative error <= 1e-4."""
    P = G.helix3d(2500, seed=33)
    r1, iters, h = 0.2, 8, 1e-3
    S0 = O.choose(P, r1)
    idx0 = chosen_indices(P, S0)
    W = np.random.default_rng(5).normal(size=S0.shape)
    _, gP, gS = adj.evolve_adjoint(P, S0, r1, iters, W)
    np.add.at(gP, idx0, gS)  # S0 = P[idx0]
    P64 = P.astype(np.float64)
    _, base_seq = forward64(P64, P64[idx0], r1, iters)
    rng = np.random.default_rng(6)
    checked = 0
    for f in rng.permutation(P.size):
        i, d = divmod(int(f), P.shape[1])
        vals, same = [], True
        for s in (1, -1):
            Pp = P64.copy()
            Pp[i, d] += s * h
            Sf, seq = forward64(Pp, Pp[idx0], r1, iters)
            same = same and all(np.array_equal(a, b) for a, b in zip(seq, base_seq))
            vals.append(float((W * Sf).sum()))
        if not same:
            continue
        fd = (vals[0] - vals[1]) / (2 * h)
        assert abs(fd - gP[i, d]) <= 1e-4 * max(abs(fd), 1e-3), (i, d, fd, gP[i, d])
        checked += 1
        if checked == 16:
            break
    assert checked == 16


def test_adjoint_config_helix_262k(adj):
    """The adjoint workload: helix N = 262,144, 20 passes, checkpoints every 5,
    W ~ N(0,1); central differences (h = 1e-3, FP64, assignments frozen) on
    64 seeded coordinates agree to 1e-4 relative."""
    P = G.helix3d(262_144)
    r1, iters, h = 0.15, 20, 1e-3
    S0 = O.choose(P, r1)
    idx0 = chosen_indices(P, S0)
    W = np.random.default_rng(2024).normal(size=S0.shape)
    Sf, gP, gS = adj.evolve_adjoint(P, S0, r1, iters, W, checkpoint_every=5)
    np.add.at(gP, idx0, gS)
    # the assignment sequence of the FP32 forward, replayed in FP64
    keys, S = [], S0.copy()
    for _ in range(iters):
        k = O.assign(P, S, r1)
        keys.append(k.astype(np.int64))
        _, sums, cnt, _, _ = O.evolve_pass(P, S, r1)
        S = S.copy()
        nz = cnt > 0
        S[nz] = (sums[nz] / cnt[nz, None].astype(np.float32)).astype(np.float32)
    assert bits_equal(S, Sf)
    P64 = P.astype(np.float64)
    rng = np.random.default_rng(7)
    for f in rng.choice(P.size, 64, replace=False):
        i, d = divmod(int(f), 3)
        vals = []
        for s in (1, -1):
            Pp = P64.copy()
            Pp[i, d] += s * h
            S_, _ = forward64(Pp, Pp[idx0], r1, iters, keys)
            vals.append(float((W * S_).sum()))
        fd = (vals[0] - vals[1]) / (2 * h)
        assert abs(fd - gP[i, d]) <= 1e-4 * max(abs(fd), 1e-6), (i, d, fd, gP[i, d])


def test_autograd_function(adj):
    torch = require_cuda()
    P = G.sine2d(3000, seed=34)
    r1 = 0.3
    S0 = O.choose(P, r1)
    idx = torch.as_tensor(chosen_indices(P, S0), device="cuda")
    Pt = torch.from_numpy(P).cuda().requires_grad_(True)
    Fn = adj.evolve_function()
    Sf = Fn.apply(Pt, idx, r1, 6)
    W = torch.randn(Sf.shape, device="cuda", generator=torch.Generator("cuda").manual_seed(1))
    (Sf * W).sum().backward()
    _, gP, gS = adj.evolve_adjoint(P, S0, r1, 6, W.double().cpu().numpy())
    np.add.at(gP, chosen_indices(P, S0), gS)
    np.testing.assert_allclose(Pt.grad.cpu().numpy(), gP.astype(np.float32), rtol=1e-6, atol=1e-7)
