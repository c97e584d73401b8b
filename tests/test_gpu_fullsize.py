"""Parity at the sizes the benchmark is quoted on, against the reference's own
serial CPU code (tests/golden/make_golden_fullsize.py made the fixtures).

  * 3D helix, N = 1,000,000 (brute force): the chosen set right after choose,
    the chosen set after each of the first five evolve passes, and the final
    ridge, bit for bit;
  * 2D spiral, N = 10,000,000, 64 x 64 tiles (tiled EXT_TILE_TREE_MIXED_RD):
    the final ridge, bit for bit; and N = 1,000,000 with 8 x 8 tiles and a
    capacity that subdivides most tiles;
  * 256 clouds of the 4,096-cloud batch (every 16th by size: 1k to 200k
    points, 2D and 3D, per-cloud r1), solved in one batched run: every cloud's
    ridge bit for bit; 16 of them also through the plain per-cloud path;
  * the adjoint workload (helix N = 262,144, 20 passes, checkpoints every 5):
    gradients against true central differences of the FP64 map with every
    assignment recomputed (h = 1e-3), on 64 seeded coordinates, 1e-4 relative.

The clouds are regenerated from their seeds; a SHA-256 of each regenerated
cloud must equal the one stored beside the reference's result.
"""
import ctypes
import hashlib
import os

import numpy as np
import pytest

import oracle as O
from gpu_util import bits_equal, require_cuda
from ridgedetection_b200 import generators as G

pytestmark = pytest.mark.gpu

GOLD = os.path.join(os.path.dirname(__file__), "golden")


@pytest.fixture(scope="module")
def rdb():
    require_cuda()
    import ridgedetection_b200 as rdb
    return rdb


def sha(P):
    return hashlib.sha256(np.ascontiguousarray(P, np.float32).tobytes()).hexdigest()


def regenerate(g):
    P = getattr(G, str(g["gen"]))(int(g["n"]), seed=int(g["seed"]))
    assert sha(P) == str(g["sha"]), "the generator no longer reproduces the fixture's cloud"
    return P


def vp(t):
    return ctypes.c_void_p(t.data_ptr())


def test_helix_1m_choose_and_first_passes(rdb):
    torch = require_cuda()
    from ridgedetection_b200 import _lib as L
    lib = L.lib()
    g = np.load(os.path.join(GOLD, "full_helix3d_1m.npz"))
    P, r1 = regenerate(g), float(g["r1"])
    st = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    dP = torch.from_numpy(P).cuda()
    dS = torch.zeros_like(dP)
    ns = ctypes.c_int64(0)
    L.check(lib.rd_choose(3, vp(dP), P.shape[0], r1, vp(dS), ctypes.byref(ns), st))
    assert bits_equal(dS[: ns.value].cpu().numpy(), g["S_choose"])
    S = dS[: ns.value].clone()
    moved = ctypes.c_int32(-1)
    for t in range(g["S_passes"].shape[0]):
        L.check(lib.rd_evolve_pass(3, vp(dP), P.shape[0], vp(S), ns.value, r1,
                                   ctypes.byref(moved), st))
        assert moved.value == 1
        assert bits_equal(S.cpu().numpy(), g["S_passes"][t]), f"pass {t + 1}"


@pytest.mark.parametrize("mode", ["graph", "host"])
def test_helix_1m_final_ridge(rdb, mode):
    g = np.load(os.path.join(GOLD, "full_helix3d_1m.npz"))
    P = regenerate(g)
    lm = rdb.LOOP_GRAPH if mode == "graph" else rdb.LOOP_HOST
    S, st = rdb.ridge_detection(P, float(g["r1"]), float(g["r2"]), loop_mode=lm)
    assert st.err_bits == 0
    assert bits_equal(S, g["S_final"]), (S.shape, g["S_final"].shape)


@pytest.mark.parametrize("name", ["full_spiral2d_10m_tiled", "full_spiral2d_1m_split"])
def test_tiled_full_size_final_ridge(rdb, name):
    g = np.load(os.path.join(GOLD, name + ".npz"))
    P = regenerate(g)
    S, st, _ = rdb.tiled_ridge_detection(P, float(g["r1"]), float(g["r2"]),
                                         int(g["max_tile_capacity"]), g["tiles_per_dim"])
    assert st.err_bits == 0
    assert bits_equal(S, g["S_final"]), (S.shape, g["S_final"].shape)


def test_batch_subset_256_clouds(rdb):
    g = np.load(os.path.join(GOLD, "batch_subset_256.npz"))
    spec = G.batch_spec()
    ids = [int(c) for c in g["cloud_ids"]]
    clouds = []
    for c, h in zip(ids, g["sha"]):
        n, dim, r1, r2, seed = spec[c]
        P = G.batch_cloud(n, dim, seed)
        assert sha(P) == str(h), c
        clouds.append((P, r1, r2))
    sizes = [P.shape[0] for P, _, _ in clouds]
    assert min(sizes) < 1100 and max(sizes) > 190_000
    ends = np.concatenate([[0], np.cumsum(g["ns"] * np.array([P.shape[1] for P, _, _ in clouds]))])
    expect = [g["S_flat"][ends[k]:ends[k + 1]].reshape(-1, clouds[k][0].shape[1])
              for k in range(len(clouds))]
    packed, descs = rdb.pack_clouds(clouds)
    b = rdb.BatchedRidgeDetection()
    counts = b.run(packed, descs)
    assert b.stats().err_bits == 0
    bad = [ids[k] for k in range(len(clouds))
           if counts[k] != expect[k].shape[0] or not bits_equal(b.chosen_points(k), expect[k])]
    b.close()
    assert not bad, f"clouds differing from the reference: {bad}"
    # the plain per-cloud path on every 16th cloud of the subset
    for k in range(0, len(clouds), 16):
        P, r1, r2 = clouds[k]
        S, _ = rdb.ridge_detection(P, r1, r2)
        assert bits_equal(S, expect[k]), ids[k]


def chosen_rows(P, S):
    """Row of P that every chosen point was copied from (choose copies the
    first point of each r1-ball in input order)."""
    first = {}
    for i, row in enumerate(P.view(np.uint32).reshape(P.shape[0], -1)):
        first.setdefault(row.tobytes(), i)
    return np.array([first[r.tobytes()] for r in S.view(np.uint32).reshape(S.shape[0], -1)])


def test_adjoint_262k_true_central_differences(rdb):
    """dL/dP from the GPU adjoint against (L(P + h e) - L(P - h e)) / 2h of the
    FP64 map with every assignment recomputed.  A coordinate is used when
    (a) the +-h runs keep every assignment of the FP64 run (its ball and
    Voronoi margins exceed the perturbation's reach), and (b) the FP32 forward
    -- whose assignments the adjoint differentiates -- and the FP64 forward
    give the clusters on the point's gradient path (its cluster at every
    pass) the same members.  FP32 and FP64 runs drift apart by a few hundred
    assignments over 20 passes on this cloud, so (b) rules out the points
    whose derivative is a different linear map in the two runs."""
    from ridgedetection_b200 import autograd as A
    P = G.helix3d(262_144)
    r1, iters, h = 0.15, 20, 1e-3
    S0 = O.choose(P, r1)
    rows = chosen_rows(P, S0)
    W = np.random.default_rng(2024).normal(size=S0.shape)
    Sf, gP, gS = A.evolve_adjoint(P, S0, r1, iters, W, checkpoint_every=5)
    np.add.at(gP, rows, gS)                       # S0 = P[rows]
    # FP32 assignment sequence of the forward the adjoint differentiates
    keys32, S = [], S0.copy()
    for _ in range(iters):
        _, sums, cnt, key, _ = O.evolve_pass(P, S, r1)
        keys32.append(key)
        S = S.copy()
        nz = cnt > 0
        S[nz] = (sums[nz] / cnt[nz, None].astype(np.float32)).astype(np.float32)
    assert bits_equal(S, Sf)
    F = O.Forward64(P, S0, r1, iters)
    agree = np.ones(P.shape[0], bool)
    for t in range(iters):
        k64, k32 = F.keys[t], keys32[t]
        diff = k64 != k32
        bad_clusters = np.zeros(S0.shape[0] + 1, bool)
        bad_clusters[k64[diff]] = True            # -1 lands in the spare last slot
        bad_clusters[k32[diff]] = True
        agree &= ~diff & ~bad_clusters[k64]
    row_of = {int(r): s for s, r in enumerate(rows)}
    rng = np.random.default_rng(7)
    checked = tried = 0
    worst = 0.0
    for f in rng.permutation(P.size):
        i, d = divmod(int(f), 3)
        if not agree[i]:
            continue
        tried += 1
        fd = F.central_difference(W, i, d, h, row_of.get(i, -1))
        if fd is None:
            continue
        err = abs(fd - gP[i, d]) / max(abs(fd), 1e-6)
        worst = max(worst, err)
        assert err <= 1e-4, (i, d, fd, gP[i, d])
        checked += 1
        if checked == 64:
            break
    assert checked == 64, (checked, tried)
    print(f"64 coordinates checked of {tried} tried; worst relative error {worst:.2e}")
