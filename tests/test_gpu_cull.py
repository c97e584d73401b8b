"""Exact chunk-box culling of the brute-force assignment (rd_set_assign_cull).

The culled assignment must give the reference's keys bit for bit: evolve runs
(rd_evolve, every pass's assignment feeds the next) are compared between the
culled kernel, the all-pairs kernel and the CPU restatement of
rd/cpu/brute_force/evolve.hpp on inputs built to stress the skip test --
points exactly r1 away, equidistant points (ties), duplicates, non-finite
coordinates, radii whose square leaves the normal range, huge coordinates --
and full ridge solves are compared with culling on and off.
"""
import ctypes

import numpy as np
import pytest

import oracle as O
from gpu_util import bits_equal, require_cuda
from ridgedetection_b200 import generators as G

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def env():
    torch = require_cuda()
    import ridgedetection_b200 as rdb
    from ridgedetection_b200 import _lib as L
    yield torch, rdb, L
    rdb.set_assign_cull(True)


def gpu_evolve(env, P, S, r1, cull):
    torch, rdb, L = env
    rdb.set_assign_cull(cull)
    try:
        P = np.ascontiguousarray(P, np.float32)
        S = np.ascontiguousarray(S, np.float32)
        dP = torch.from_numpy(P).cuda()
        dS = torch.from_numpy(S.copy()).cuda()
        passes = ctypes.c_int64(0)
        st = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
        L.check(L.lib().rd_evolve(P.shape[1], ctypes.c_void_p(dP.data_ptr()), P.shape[0],
                                  ctypes.c_void_p(dS.data_ptr()), S.shape[0], float(r1),
                                  ctypes.byref(passes), st))
        return dS.cpu().numpy(), passes.value
    finally:
        rdb.set_assign_cull(True)


def _lattice(dim, side, h, jitter, rng):
    g = np.stack(np.meshgrid(*[np.arange(side, dtype=np.float32) * np.float32(h)] * dim,
                             indexing="ij"), -1).reshape(-1, dim)
    if jitter:
        # +-1 ulp moves: distances land just inside, on, or just outside r1
        steps = rng.integers(-1, 2, size=g.shape)
        g = np.where(steps > 0, np.nextafter(g, np.float32(np.inf)),
                     np.where(steps < 0, np.nextafter(g, np.float32(-np.inf)), g)).astype(np.float32)
    return g.astype(np.float32)


def _cases():
    r = np.random.default_rng(11)
    cases = {}
    # lattice points at spacing h = r1: every point is exactly r1 from its
    # lattice neighbours, chosen points on the lattice too (ties everywhere)
    for dim in (2, 3):
        side = 40 if dim == 2 else 14
        P = _lattice(dim, side, 0.25, False, r)
        cases[f"lattice_exact_{dim}d"] = (P, P[r.permutation(len(P))[: len(P) // 7]], 0.25)
        Pj = _lattice(dim, side, 0.25, True, r)
        cases[f"lattice_ulp_{dim}d"] = (Pj, P[r.permutation(len(P))[: len(P) // 5]], 0.25)
    # duplicates: every point three times, chosen points duplicated too
    base = r.normal(size=(3000, 2)).astype(np.float32)
    P = np.repeat(base, 3, axis=0)
    S = np.repeat(base[:200], 2, axis=0)
    cases["duplicates"] = (P, S, 0.3)
    # non-finite cloud points and one non-finite chosen point
    P = (r.normal(size=(20000, 3)) * 2).astype(np.float32)
    P[::997, 0] = np.nan
    P[5::1009, 1] = np.inf
    P[7::1013, 2] = -np.inf
    S = O.choose(np.nan_to_num(P[:5000], nan=0.0, posinf=0.0, neginf=0.0), 0.5)
    S = np.concatenate([S, np.array([[np.inf, 0.0, 0.0]], np.float32), S[:3]])
    cases["nonfinite"] = (P, S, 0.5)
    # radii whose square leaves [1e-30, 1e30] (no skipping) and radii just
    # inside that range (skipping, with subnormal or huge distance terms)
    for name, scale, r1 in (("subnormal_r1", 1e-19, 3e-20), ("small_r1", 1e-14, 2e-15),
                            ("large_r1", 1e18, 3e17), ("big_r1", 1e15, 5e14)):
        P = (r.normal(size=(8000, 2)) * scale).astype(np.float32)
        cases[name] = (P, O.choose(P, r1)[:300], r1)
    # large coordinates with a moderate radius (wide chunk boxes in cell
    # units, wrapped Morton cells)
    P = (r.uniform(-1, 1, size=(30000, 3)) * np.array([5e6, 10.0, 10.0])).astype(np.float32)
    cases["far_apart"] = (P, O.choose(P, 2.0)[:400], 2.0)
    # curve with clutter, several radii
    for r1 in (0.05, 0.2, 0.6):
        P = G.sine2d(15000, seed=5)
        P = np.concatenate([P, r.uniform(-1, 11, size=(1500, 2)).astype(np.float32)])
        cases[f"sine_clutter_r{r1}"] = (P, O.choose(P, r1), r1)
    return cases


CASES = _cases()


@pytest.mark.parametrize("name", sorted(CASES))
def test_culled_evolve_matches_all_pairs_and_oracle(env, name):
    P, S0, r1 = CASES[name]
    S_on, p_on = gpu_evolve(env, P, S0, r1, True)
    S_off, p_off = gpu_evolve(env, P, S0, r1, False)
    assert p_on == p_off
    assert bits_equal(S_on, S_off), name
    S_ref, p_ref = O.evolve(P, S0, r1)
    assert p_on == p_ref
    assert bits_equal(S_on, S_ref), name


@pytest.mark.parametrize("kind", ["helix", "sine"])
def test_culled_ridge_equals_all_pairs(env, kind):
    torch, rdb, L = env
    if kind == "helix":
        P, r1, r2 = G.helix3d(200_000, seed=3), 0.15, 0.3
    else:
        P, r1, r2 = G.sine2d(60_000, seed=4), 0.3, 0.6
    rdb.set_assign_cull(False)
    try:
        S_off, st_off = rdb.ridge_detection(P, r1, r2)
    finally:
        rdb.set_assign_cull(True)
    S_on, st_on = rdb.ridge_detection(P, r1, r2)
    assert bits_equal(S_on, S_off)
    assert st_on.evolve_passes == st_off.evolve_passes
    assert st_on.pairs == st_off.pairs


def test_cull_switch_roundtrip(env):
    torch, rdb, L = env
    assert rdb.get_assign_cull()
    rdb.set_assign_cull(False)
    assert not rdb.get_assign_cull()
    rdb.set_assign_cull(True)
    assert rdb.get_assign_cull()
