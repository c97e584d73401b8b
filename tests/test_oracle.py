"""The CPU restatement (oracle/rd_oracle.c) against the reference's own outputs.

Fixtures in tests/golden/ were produced by the reference's CPU code compiled from
its sources (tests/golden/make_golden.py); every comparison here is bit for bit.
"""
import glob
import os

import numpy as np
import pytest

import oracle as O

GOLD = os.path.join(os.path.dirname(__file__), "golden")
BF = sorted(glob.glob(os.path.join(GOLD, "bf_*.npz")))
TILED = sorted(glob.glob(os.path.join(GOLD, "tiled_*.npz")))


def bits_equal(a, b):
    a = np.ascontiguousarray(a, np.float32)
    b = np.ascontiguousarray(b, np.float32)
    return a.shape == b.shape and np.array_equal(a.view(np.uint32), b.view(np.uint32))


@pytest.mark.parametrize("path", BF, ids=[os.path.basename(p) for p in BF])
def test_bf_steps_match_reference(path):
    g = np.load(path)
    P, r1, r2 = g["P"], float(g["r1"]), float(g["r2"])
    S0 = O.choose(P, r1)
    assert bits_equal(S0, g["S_choose"])
    S1, sums, cnt, _key, cont = O.evolve_pass(P, S0, r1)
    assert bits_equal(S1, g["S_pass1"])
    assert bits_equal(sums, g["sums_pass1"])
    assert np.array_equal(cnt, g["cnt_pass1"])
    assert cont == int(g["cont_pass1"])
    Se, passes = O.evolve(P, S0, r1)
    assert passes >= 1
    assert bits_equal(Se, g["S_evolved"])
    assert bits_equal(O.decimate(Se, r2), g["S_decimated"])
    Sd, seg = O.decimate_seg(Se, g["seg_in"], r2)
    assert bits_equal(Sd, g["S_decimated_nocopy"])
    assert np.array_equal(seg, g["seg_out"])


@pytest.mark.parametrize("path", BF, ids=[os.path.basename(p) for p in BF])
def test_bf_pipeline_matches_reference(path):
    g = np.load(path)
    S, st = O.ridge_bf(g["P"], float(g["r1"]), float(g["r2"]))
    assert bits_equal(S, g["S_final"])
    assert st.ns_choose == g["S_choose"].shape[0]


@pytest.mark.parametrize("path", TILED, ids=[os.path.basename(p) for p in TILED])
def test_tiled_pipeline_matches_reference(path):
    g = np.load(path)
    S, _st, nl = O.ridge_tiled(g["P"], float(g["r1"]), float(g["r2"]),
                               int(g["max_tile_capacity"]), g["tiles_per_dim"])
    assert nl >= 1
    assert bits_equal(S, g["S_final"])


def test_hausdorff_basic():
    A = np.array([[0, 0], [1, 0]], np.float32)
    B = np.array([[0, 0], [1, 0], [1, 2]], np.float32)
    assert O.hausdorff(A, A) == 0.0
    assert abs(O.hausdorff(A, B) - 2.0) < 1e-12


def test_adjoint_oracle_matches_finite_differences():
    """FP64 reverse pass vs central differences of the same forward with the
    assignment frozen (the forward is then affine in P, so FD is exact)."""
    from ridgedetection_b200 import generators as G
    P = G.helix3d(3000, seed=21)
    r1 = 0.2
    S0 = O.choose(P, r1)
    rng = np.random.default_rng(5)
    W = rng.normal(size=S0.shape)
    iters = 6
    gP, gS0, Sf = O.evolve_adjoint(P, S0, r1, iters, W)
    # frozen-assignment FP64 forward
    keys = []
    S = S0.astype(np.float32).copy()
    for _ in range(iters):
        k = O.assign(P, S, r1)
        keys.append(k)
        _, sums, cnt, _, _ = O.evolve_pass(P, S, r1)
        nz = cnt > 0
        S = S.copy()
        S[nz] = (sums[nz] / cnt[nz, None].astype(np.float32)).astype(np.float32)
    assert np.array_equal(S, Sf)

    def fwd64(Pd, S0d):
        Sd = S0d.copy()
        for k in keys:
            out = Sd.copy()
            for c in np.unique(k[k >= 0]):
                out[c] = Pd[k == c].mean(axis=0)
            Sd = out
        return float((W * Sd).sum())
    P64, S064 = P.astype(np.float64), S0.astype(np.float64)
    h = 1e-3
    idx = rng.choice(P.shape[0] * 3, 12, replace=False)
    for f in idx:
        i, d = divmod(int(f), 3)
        Pp, Pm = P64.copy(), P64.copy()
        Pp[i, d] += h
        Pm[i, d] -= h
        fd = (fwd64(Pp, S064) - fwd64(Pm, S064)) / (2 * h)
        assert abs(fd - gP[i, d]) <= 1e-8 + 1e-6 * abs(fd)


def _order_cases():
    from ridgedetection_b200 import generators as G
    r = np.random.default_rng(1)
    S1, _ = O.ridge_bf(G.sine2d(20000, seed=3), 0.3, 0.6)
    return [("sine_ridge", S1, 0.6),
            ("random_2d", r.random((3000, 2)).astype(np.float32), 0.03),
            ("random_3d", r.random((2000, 3)).astype(np.float32), 0.08),
            ("duplicates", np.repeat(r.random((50, 3)).astype(np.float32), 4, axis=0), 0.05),
            ("one", np.zeros((1, 2), np.float32), 0.1),
            ("empty", np.zeros((0, 2), np.float32), 0.1)]


@pytest.mark.parametrize("case", _order_cases(), ids=lambda c: c[0])
def test_order_restatement_matches_reference(case):
    """rd_oracle.c rdo_order == the reference's own rd::orderSamples."""
    if O.ref(False) is None:
        pytest.skip("oracle/_ref not built")
    _, S, r2 = case
    a, b = O.order(S, r2), O.ref_order(S, r2)
    assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])
    assert sorted(a[0].tolist()) == list(range(S.shape[0]))   # a permutation


def _quality_sets():
    r = np.random.default_rng(5)
    t = r.uniform(0, 6 * np.pi, 20000)
    ideal = np.stack([0.5 * t * np.cos(t), 0.5 * t * np.sin(t)], 1).astype(np.float32)
    S, _, _ = O.ridge_tiled(O_gen_spiral(), 0.2, 0.4, 100_001, (16, 16))
    return [("ridge_vs_spiral", S, ideal),
            ("random3d", r.normal(size=(700, 3)).astype(np.float32),
             r.normal(size=(3000, 3)).astype(np.float32)),
            ("single", np.ones((1, 2), np.float32), np.zeros((5, 2), np.float32))]


def O_gen_spiral():
    from ridgedetection_b200 import generators as G
    return G.spiral2d(100_000, seed=6)


@pytest.mark.parametrize("case", _quality_sets(), ids=lambda c: c[0])
def test_quality_restatement_matches_reference(case):
    """rd_oracle.c float Hausdorff / distance stats / segment distance == the
    reference's own RDAssessmentQuality<float>."""
    if O.ref(False) is None:
        pytest.skip("oracle/_ref not built")
    _, T, I = case
    for which in ("hausdorff", "stats", "segment"):
        a = O.quality(T, I, which)
        b = O.quality(T, I, which, use_ref=True)
        assert np.array_equal(np.float32(a), np.float32(b)), (which, a, b)
    assert O.quality(np.zeros((0, 2), np.float32), I, "hausdorff") == -1.0


# --------------------------------------------------------------------------
# full-size fixtures (tests/golden/make_golden_fullsize.py): the clouds are
# regenerated from their seeds and checked against the stored SHA-256
# --------------------------------------------------------------------------

def _regenerate(g):
    import hashlib

    from ridgedetection_b200 import generators as G
    P = getattr(G, str(g["gen"]))(int(g["n"]), seed=int(g["seed"]))
    assert hashlib.sha256(P.tobytes()).hexdigest() == str(g["sha"])
    return P


def test_full_helix_1m_choose_and_first_passes_match_reference():
    g = np.load(os.path.join(GOLD, "full_helix3d_1m.npz"))
    P, r1 = _regenerate(g), float(g["r1"])
    S = O.choose(P, r1)
    assert bits_equal(S, g["S_choose"])
    for t in range(g["S_passes"].shape[0]):
        S, _, _, _, cont = O.evolve_pass(P, S, r1)
        assert cont == 1 and bits_equal(S, g["S_passes"][t]), t


def test_full_tiled_1m_split_matches_reference():
    g = np.load(os.path.join(GOLD, "full_spiral2d_1m_split.npz"))
    P = _regenerate(g)
    S, _, n_leaves = O.ridge_tiled(P, float(g["r1"]), float(g["r2"]),
                                   int(g["max_tile_capacity"]), g["tiles_per_dim"])
    assert n_leaves > 64   # the capacity subdivided tiles
    assert bits_equal(S, g["S_final"])


def test_batch_subset_small_clouds_match_reference():
    """The clouds of the 256-cloud batch fixture with fewer than 5,000 points
    (the larger ones are checked on the GPU against the same fixture)."""
    import hashlib

    from ridgedetection_b200 import generators as G
    g = np.load(os.path.join(GOLD, "batch_subset_256.npz"))
    spec = G.batch_spec()
    off, checked = 0, 0
    for k, c in enumerate(g["cloud_ids"]):
        n, dim, r1, r2, seed = spec[int(c)]
        m = int(g["ns"][k]) * dim
        if n < 5000:
            P = G.batch_cloud(n, dim, seed)
            assert hashlib.sha256(P.tobytes()).hexdigest() == str(g["sha"][k])
            S, _ = O.ridge_bf(P, r1, r2)
            assert bits_equal(S, g["S_flat"][off:off + m].reshape(-1, dim)), int(c)
            checked += 1
        off += m
    assert checked >= 30


@pytest.mark.parametrize("dim", [1, 4])
def test_restatement_matches_reference_in_other_dims(dim):
    """The restatement against the reference's own serial code in 1 and 4
    dimensions (the CPU API takes the dimension at run time)."""
    r = np.random.default_rng(dim)
    if dim == 1:
        P = np.sort(r.normal(0, 2, 3000))[r.permutation(3000)][:, None].astype(np.float32)
        r1, r2 = 0.1, 0.2
    else:
        t = r.uniform(0, 6 * np.pi, 3000)
        P = np.stack([np.cos(t), np.sin(t), 0.15 * t, 0.3 * np.sin(2 * t)], 1)
        P = (P + r.normal(0, 0.05, P.shape)).astype(np.float32)
        r1, r2 = 0.2, 0.4
    S, _ = O.ridge_bf(P, r1, r2)
    assert bits_equal(S, O.ref_ridge_bf(P, r1, r2))
    assert bits_equal(O.choose(P, r1), O.ref_choose(P, r1))
