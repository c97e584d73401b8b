"""Generate the golden fixtures in tests/golden/ from the reference's own CPU code.

The reference has no golden vectors of its own (its generators are unseeded and
the data files it names are not in its repository), so the fixtures are made by
running the reference's CPU implementation, compiled from its sources by
`make -C oracle ref REF=<checkout>/ridge_detection` into oracle/_ref/librdref.so
(serial build), on seeded inputs.  Each fixture stores the input cloud and the
reference's outputs; the tests then check the plain-C restatement
(oracle/rd_oracle.c) and the GPU path against them bit for bit.

Run from the repository root:  python tests/golden/make_golden.py
"""
from __future__ import annotations

import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

import oracle as O  # noqa: E402
from ridgedetection_b200 import generators as G  # noqa: E402

OUT = os.path.dirname(os.path.abspath(__file__))


def lattice_ties(n_side=12, spacing=0.25):
    """Points on an exact binary-fraction lattice: many exactly equal distances,
    so argmin ties (lowest index must win) and threshold equalities occur."""
    xs = np.arange(n_side, dtype=np.float32) * np.float32(spacing)
    P = np.stack(np.meshgrid(xs, xs, indexing="ij"), -1).reshape(-1, 2)
    rng = np.random.default_rng(11)
    return np.ascontiguousarray(P[rng.permutation(P.shape[0])], dtype=np.float32)


CASES = {
    # name: (cloud, r1, r2)
    "sine2d_3k": (lambda: G.sine2d(3000, seed=7), 0.3, 0.6),
    "sine2d_20k": (lambda: G.sine2d(20000), 0.3, 0.6),
    "helix3d_5k": (lambda: G.helix3d(5000, seed=9), 0.2, 0.4),
    "helix3d_20k": (lambda: G.helix3d(20000), 0.15, 0.3),
    "lattice_ties": (lattice_ties, 0.25, 0.5),
    "tiny_2": (lambda: np.array([[0, 0], [1, 1]], np.float32), 0.3, 0.6),
    "tiny_1": (lambda: np.array([[0.5, -0.5, 2.0]], np.float32), 0.3, 0.6),
    "dup_points": (lambda: np.repeat(G.sine2d(40, seed=3), 5, axis=0), 0.3, 0.6),
    "huge_r1": (lambda: G.helix3d(2000, seed=4), 100.0, 200.0),
    "tiny_r1": (lambda: G.sine2d(600, seed=5), 1e-4, 2e-4),
}

TILED = {
    # name: (cloud, r1, r2, max_tile_capacity, tiles_per_dim)
    "spiral2d_20k_flat": (lambda: G.spiral2d(20000, seed=3), 0.2, 0.4, 20001, (8, 8)),
    "spiral2d_20k_split": (lambda: G.spiral2d(20000, seed=3), 0.2, 0.4, 800, (4, 4)),
    "helix3d_20k_tiled": (lambda: G.helix3d(20000, seed=5), 0.15, 0.3, 3000, (3, 3, 2)),
    "sine2d_5k_tiled": (lambda: G.sine2d(5000, seed=8), 0.3, 0.6, 5001, (5, 2)),
}


def main():
    if O.ref() is None:
        raise SystemExit("oracle/_ref/librdref.so missing: run "
                         "`make -C oracle ref REF=<checkout>/ridge_detection` first")
    for name, (gen, r1, r2) in CASES.items():
        P = gen()
        S_choose = O.ref_choose(P, r1)
        S1, sums1, cnt1, cont1 = O.ref_evolve_pass(P, S_choose, r1)
        S_evolved = O.ref_evolve(P, S_choose, r1)
        S_dec = O.ref_decimate(S_evolved, r2)
        # decimateNoCopy over three ragged segments of the same evolved set
        ns = S_evolved.shape[0]
        seg = np.array([ns // 3, 0, ns - ns // 3], np.int64)
        S_dnc, seg_out = O.ref_decimate_nocopy(S_evolved, seg, r2)
        S_final = O.ref_ridge_bf(P, r1, r2)
        np.savez_compressed(
            os.path.join(OUT, f"bf_{name}.npz"), P=P, r1=np.float32(r1), r2=np.float32(r2),
            S_choose=S_choose, S_pass1=S1, sums_pass1=sums1, cnt_pass1=cnt1,
            cont_pass1=np.int32(cont1), S_evolved=S_evolved, S_decimated=S_dec,
            seg_in=seg, S_decimated_nocopy=S_dnc, seg_out=seg_out, S_final=S_final)
        print(f"bf_{name}: np={P.shape[0]} ns_choose={S_choose.shape[0]} "
              f"ns_final={S_final.shape[0]}")
    for name, (gen, r1, r2, cap, tpd) in TILED.items():
        P = gen()
        S, _ = O.ref_ridge_tiled(P, r1, r2, cap, tpd)
        np.savez_compressed(
            os.path.join(OUT, f"tiled_{name}.npz"), P=P, r1=np.float32(r1), r2=np.float32(r2),
            max_tile_capacity=np.int64(cap), tiles_per_dim=np.array(tpd, np.int64), S_final=S)
        print(f"tiled_{name}: np={P.shape[0]} ns_final={S.shape[0]}")


if __name__ == "__main__":
    main()
