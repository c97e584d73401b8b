"""The skip test of the culled assignment (k_assign_cull, rd_kernels.cu), in
float32 on the CPU: whenever the computed squared gap g2 between a chosen
point s and the bounding box of a group of points exceeds
thr = r1^2 (1 + 2^-10) (rounded up), every distance the reference computes
from s to a point of the group (t = s - p; acc += t*t, rd/cpu/brute_force/
evolve.hpp:54-62) exceeds r1^2 -- so a skipped chosen point can never be the
nearest one within r1, nor tie with it.  numpy's float32 operations round to
nearest like the device's __fsub_rn/__fmul_rn/__fadd_rn; np.fmax ignores a
NaN operand like fmaxf."""
import numpy as np
import pytest

F = np.float32


def box_gap2(s, lo, hi):
    """Per row of s (m x DIM): the kernel's box_gap2, operation by operation."""
    g2 = np.zeros(s.shape[0], F)
    for d in range(s.shape[1]):
        gap = np.fmax(np.fmax(F(lo[d]) - s[:, d], s[:, d] - F(hi[d])), F(0))
        g2 = (g2 + (gap * gap).astype(F)).astype(F)
    return g2


def sqdist(s, P):
    """Reference distance from every s (m x DIM) to every P (n x DIM): m x n."""
    t = (s[:, None, 0] - P[None, :, 0]).astype(F)
    acc = (t * t).astype(F)
    for d in range(1, s.shape[1]):
        t = (s[:, None, d] - P[None, :, d]).astype(F)
        acc = (acc + (t * t).astype(F)).astype(F)
    return acc


def threshold(rsq):
    """__fmul_ru(rsq, 1 + 2^-10): the product is exact in float64."""
    x = float(rsq) * 1.0009765625
    f = F(x)
    return f if float(f) >= x else np.nextafter(f, F(np.inf))


def _case(rng, dim):
    r1 = F(10.0 ** rng.uniform(-13, 13))
    rsq = F(r1 * r1)
    center = (rng.normal(size=dim) * 10.0 ** rng.uniform(-2, 6) * float(r1)).astype(F)
    n = int(rng.integers(1, 64))
    P = (center + rng.uniform(-1, 1, size=(n, dim)) * rng.uniform(0, 3) * float(r1)).astype(F)
    lo, hi = P.min(0), P.max(0)
    # chosen points near the sphere of radius r1 around the box's nearest
    # point: along an axis, towards a corner, or in a random direction, with
    # relative offsets of a few ulps up to 1e-3
    m = 256
    base = P[rng.integers(0, n, size=m)].astype(np.float64)
    kind = rng.integers(0, 3, size=m)
    dirs = rng.normal(size=(m, dim))
    axis = np.zeros((m, dim))
    axis[np.arange(m), rng.integers(0, dim, size=m)] = rng.choice([-1.0, 1.0], size=m)
    corner = rng.choice([-1.0, 1.0], size=(m, dim))
    dirs = np.where(kind[:, None] == 0, axis, np.where(kind[:, None] == 1, corner, dirs))
    dirs /= np.linalg.norm(dirs, axis=1, keepdims=True)
    # along an axis, start from the group's extreme point on that side: the
    # gap to the box is then r1 * scale up to rounding, right at the threshold
    for i in np.flatnonzero(kind == 0):
        d = int(np.flatnonzero(axis[i])[0])
        j = int(np.argmax(P[:, d]) if axis[i, d] > 0 else np.argmin(P[:, d]))
        base[i] = P[j]
    scale = 1.0 + rng.choice([-1.0, 1.0], size=m) * 10.0 ** rng.uniform(-9, -3, size=m)
    s = (base + dirs * float(r1) * scale[:, None]).astype(F)
    # and some snapped one ulp either way
    bump = rng.integers(-1, 2, size=s.shape)
    s = np.where(bump > 0, np.nextafter(s, F(np.inf)),
                 np.where(bump < 0, np.nextafter(s, F(-np.inf)), s)).astype(F)
    return P, lo, hi, s, rsq


@pytest.mark.parametrize("dim", [2, 3])
def test_skipped_chosen_points_are_beyond_r1(dim):
    rng = np.random.default_rng(1234 + dim)
    skipped = 0
    for _ in range(400):
        P, lo, hi, s, rsq = _case(rng, dim)
        thr = threshold(rsq)
        skip = box_gap2(s, lo, hi) > thr
        if not skip.any():
            continue
        skipped += int(skip.sum())
        acc = sqdist(s[skip], P)
        assert np.all(acc > rsq), (rsq, thr, acc.min())
    assert skipped > 1000  # the cases do reach the boundary


def test_kept_when_a_point_is_within_r1():
    """The converse check on the same cases: a chosen point with some group
    point within r1 (acc <= r1^2) is never skipped."""
    rng = np.random.default_rng(99)
    within = 0
    for _ in range(400):
        dim = int(rng.integers(2, 4))
        P, lo, hi, s, rsq = _case(rng, dim)
        near = (sqdist(s, P) <= rsq).any(1)
        within += int(near.sum())
        assert not np.any(near & (box_gap2(s, lo, hi) > threshold(rsq)))
    assert within > 1000


def test_nan_never_skips_and_inf_is_beyond():
    lo, hi = np.array([0.0, 0.0], F), np.array([1.0, 1.0], F)
    s = np.array([[np.nan, 5.0], [np.nan, np.nan], [np.inf, 0.5], [-np.inf, 0.5]], F)
    g2 = box_gap2(s, lo, hi)
    thr = threshold(F(0.25))
    assert g2[1] == 0.0 and not g2[1] > thr        # all-NaN: gap 0, kept
    assert np.isinf(g2[2]) and np.isinf(g2[3])     # infinite gap: skipped, and the
    P = np.array([[0.0, 0.0], [1.0, 1.0]], F)      # reference distance is inf too
    assert np.all(np.isinf(sqdist(s[2:], P)))
