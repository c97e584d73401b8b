"""CPU checker for the ridge-detection path -- TEST INFRASTRUCTURE ONLY.

Two ctypes-loaded libraries live here:
  * ``librdoracle.so``  -- the plain-C restatement of the reference path
    (``rd_oracle.c``), built by ``oracle/Makefile``;
  * ``_ref/librdref.so`` / ``_ref/librdref_omp.so`` -- the reference's own CPU
    code compiled from its sources through ``ref_shim.cpp`` (present only when
    the reference checkout was available at build time).

Only tests/, ``__graft_entry__.smoke()`` and the CPU-baseline leg of bench.py use
this package, and only to check or to time the CPU side; the product
(``ridgedetection_b200``) never imports it.
"""
from __future__ import annotations

import ctypes
import os
from typing import Optional

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_F = ctypes.POINTER(ctypes.c_float)
_D = ctypes.POINTER(ctypes.c_double)
_I32 = ctypes.POINTER(ctypes.c_int32)
_I64 = ctypes.POINTER(ctypes.c_int64)
_i64 = ctypes.c_int64
_int = ctypes.c_int
_flt = ctypes.c_float


class Stats(ctypes.Structure):
    _fields_ = [("outer_iters", ctypes.c_int64), ("evolve_passes", ctypes.c_int64),
                ("pairs", ctypes.c_double), ("ns_choose", ctypes.c_int64)]


def _fp(a):
    return a.ctypes.data_as(_F)


def _load(path):
    if not os.path.exists(path):
        raise FileNotFoundError(f"{path} is missing; run `make -C oracle`")
    return ctypes.CDLL(path)


_lib = None
_ref = {}


def lib():
    """The plain-C restatement (rd_oracle.c)."""
    global _lib
    if _lib is None:
        L = _load(os.path.join(_HERE, "librdoracle.so"))
        L.rdo_choose.restype = _i64
        L.rdo_choose.argtypes = [_F, _i64, _int, _flt, _F]
        L.rdo_assign.restype = None
        L.rdo_assign.argtypes = [_F, _i64, _F, _i64, _int, _flt, _I32]
        L.rdo_accumulate.restype = None
        L.rdo_accumulate.argtypes = [_F, _i64, _I32, _i64, _int, _F, _I32]
        L.rdo_shift.restype = _int
        L.rdo_shift.argtypes = [_F, _F, _I32, _i64, _int]
        L.rdo_evolve_pass.restype = _int
        L.rdo_evolve_pass.argtypes = [_F, _i64, _F, _i64, _int, _flt, _F, _I32, _I32]
        L.rdo_evolve.restype = _i64
        L.rdo_evolve.argtypes = [_F, _i64, _F, _i64, _int, _flt, _i64, _D]
        L.rdo_decimate.restype = _i64
        L.rdo_decimate.argtypes = [_F, _i64, _int, _flt]
        L.rdo_decimate_seg.restype = _i64
        L.rdo_decimate_seg.argtypes = [_F, _i64, _I64, _int, _flt]
        L.rdo_ridge_bf.restype = _i64
        L.rdo_ridge_bf.argtypes = [_F, _i64, _int, _flt, _flt, _F, ctypes.POINTER(Stats)]
        L.rdo_ridge_tiled.restype = _i64
        L.rdo_ridge_tiled.argtypes = [_F, _i64, _int, _flt, _flt, _i64, _I64, _F, _I64,
                                      ctypes.POINTER(Stats)]
        L.rdo_hausdorff.restype = ctypes.c_double
        L.rdo_hausdorff.argtypes = [_F, _i64, _F, _i64, _int]
        L.rdo_ridge_tiled_policy.restype = _i64
        L.rdo_ridge_tiled_policy.argtypes = [_F, _i64, _int, _flt, _flt, _i64, _I64, _int, _F,
                                             ctypes.POINTER(ctypes.c_int64),
                                             ctypes.POINTER(Stats)]
        L.rdo_hausdorff_f32.restype = _flt
        L.rdo_hausdorff_f32.argtypes = [_F, _i64, _F, _i64, _int]
        L.rdo_distance_stats_f32.restype = None
        L.rdo_distance_stats_f32.argtypes = [_F, _i64, _F, _i64, _int, _F]
        L.rdo_segment_hausdorff_f32.restype = _flt
        L.rdo_segment_hausdorff_f32.argtypes = [_F, _i64, _int]
        L.rdo_order.restype = _i64
        L.rdo_order.argtypes = [_F, _i64, _int, _flt, _I32, _I32]
        L.rdo_forward64.restype = _int
        L.rdo_forward64.argtypes = [_D, _i64, _D, _i64, _int, ctypes.c_double, _int, _D, _I32,
                                    _I32]
        L.rdo_fd64.restype = _int
        L.rdo_fd64.argtypes = [_D, _i64, _D, _I32, _I32, _i64, _int, ctypes.c_double, _int, _D,
                               _i64, _int, _i64, ctypes.c_double, _D]
        L.rdo_evolve_adjoint.restype = _int
        L.rdo_evolve_adjoint.argtypes = [_F, _i64, _F, _i64, _int, _flt, _int, _D, _D, _D, _F]
        _lib = L
    return _lib


def ref(openmp: bool = False):
    """The reference's own CPU code (serial or OpenMP build), or None."""
    name = "librdref_omp.so" if openmp else "librdref.so"
    if name not in _ref:
        path = os.path.join(_HERE, "_ref", name)
        if not os.path.exists(path):
            _ref[name] = None
        else:
            L = ctypes.CDLL(path)
            L.ref_choose.restype = _i64
            L.ref_choose.argtypes = [_F, _i64, _int, _flt, _F]
            L.ref_evolve_pass.restype = _int
            L.ref_evolve_pass.argtypes = [_F, _i64, _F, _i64, _int, _flt, _F, _I32]
            L.ref_evolve.restype = None
            L.ref_evolve.argtypes = [_F, _i64, _F, _i64, _int, _flt, _int]
            L.ref_decimate.restype = _i64
            L.ref_decimate.argtypes = [_F, _i64, _int, _flt]
            L.ref_decimate_nocopy.restype = _i64
            L.ref_decimate_nocopy.argtypes = [_F, _i64, _I64, _int, _flt]
            L.ref_bf_ridge.restype = _i64
            L.ref_bf_ridge.argtypes = [_F, _i64, _int, _flt, _flt, _F, _int]
            L.ref_load_text.restype = _i64
            L.ref_load_text.argtypes = [ctypes.c_char_p, ctypes.c_char_p, _F, _i64,
                                        ctypes.POINTER(ctypes.c_int)]
            L.ref_hausdorff_f32.restype = _flt
            L.ref_hausdorff_f32.argtypes = [_F, _i64, _F, _i64, _int]
            L.ref_distance_stats_f32.restype = None
            L.ref_distance_stats_f32.argtypes = [_F, _i64, _F, _i64, _int, _F]
            L.ref_segment_hausdorff_f32.restype = _flt
            L.ref_segment_hausdorff_f32.argtypes = [_F, _i64, _int]
            L.ref_order.restype = _i64
            L.ref_order.argtypes = [_F, _i64, _int, _flt, _I32, _I32]
            L.ref_tiled_ridge.restype = _i64
            L.ref_tiled_ridge.argtypes = [_F, _i64, _int, _flt, _flt, _i64, _I64, _int, _int,
                                          _F, _F]
            L.ref_max_threads.restype = _int
            L.ref_evolve_passes_omp.restype = _int
            L.ref_evolve_passes_omp.argtypes = [_F, _i64, _F, _i64, _int, _flt, _int, _int]
            _ref[name] = L
    return _ref[name]


def _f32(P):
    return np.ascontiguousarray(P, dtype=np.float32)


# --------------------------------------------------------------------------
# restatement wrappers
# --------------------------------------------------------------------------

def choose(P, r1):
    P = _f32(P)
    n, dim = P.shape
    S = np.zeros_like(P)
    ns = lib().rdo_choose(_fp(P), n, dim, r1, _fp(S))
    return S[:ns].copy()


def assign(P, S, r1):
    P, S = _f32(P), _f32(S)
    key = np.empty(P.shape[0], dtype=np.int32)
    lib().rdo_assign(_fp(P), P.shape[0], _fp(S), S.shape[0], P.shape[1], r1,
                     key.ctypes.data_as(_I32))
    return key


def evolve_pass(P, S, r1):
    """One pass; returns (S_new, sums, counts, keys, cont)."""
    P, S = _f32(P), _f32(S).copy()
    ns, dim = S.shape
    sums = np.zeros((ns, dim), np.float32)
    cnt = np.zeros(ns, np.int32)
    key = np.zeros(P.shape[0], np.int32)
    cont = lib().rdo_evolve_pass(_fp(P), P.shape[0], _fp(S), ns, dim, r1, _fp(sums),
                                 cnt.ctypes.data_as(_I32), key.ctypes.data_as(_I32))
    return S, sums, cnt, key, cont


def evolve(P, S, r1, max_passes=0):
    P, S = _f32(P), _f32(S).copy()
    pairs = ctypes.c_double(0)
    passes = lib().rdo_evolve(_fp(P), P.shape[0], _fp(S), S.shape[0], P.shape[1], r1,
                              max_passes, ctypes.byref(pairs))
    return S, passes


def decimate(S, r2):
    S = _f32(S).copy()
    ns = lib().rdo_decimate(_fp(S), S.shape[0], S.shape[1], r2)
    return S[:ns].copy()


def decimate_seg(S, seg_cnt, r2):
    S = _f32(S).copy()
    seg = np.ascontiguousarray(seg_cnt, dtype=np.int64).copy()
    ns = lib().rdo_decimate_seg(_fp(S), len(seg), seg.ctypes.data_as(_I64), S.shape[1], r2)
    return S[:ns].copy(), seg


def ridge_bf(P, r1, r2):
    P = _f32(P)
    S = np.zeros_like(P)
    st = Stats()
    ns = lib().rdo_ridge_bf(_fp(P), P.shape[0], P.shape[1], r1, r2, _fp(S), ctypes.byref(st))
    return S[:ns].copy(), st


def ridge_tiled_local(P, r1, r2, max_tile_capacity, tiles_per_dim, refine=False):
    """RD_LOCAL tile policy: a full ridge detection inside every leaf."""
    P = _f32(P)
    S = np.zeros_like(P)
    tpd = np.ascontiguousarray(tiles_per_dim, dtype=np.int64)
    nl = ctypes.c_int64(0)
    st = Stats()
    ns = lib().rdo_ridge_tiled_policy(_fp(P), P.shape[0], P.shape[1], r1, r2, max_tile_capacity,
                                      tpd.ctypes.data_as(_I64), 1, _fp(S), ctypes.byref(nl),
                                      ctypes.byref(st))
    if ns < 0:
        raise RuntimeError("tile subdivision did not terminate")
    S = S[:ns].copy()
    if refine and ns > 0:
        S = decimate(S, r2)
        S, _ = evolve(P, S, r1)
    return S, st, nl.value


def ridge_tiled(P, r1, r2, max_tile_capacity, tiles_per_dim, refine=False):
    """EXT_TILE_TREE_MIXED_RD; with refine, the end-phase refinement of
    rd_tiled.hpp:1386-1419 (brute-force decimate, then evolve of the whole
    cloud) composed of the restated decimate and evolve."""
    if refine:
        S, st, nl = ridge_tiled(P, r1, r2, max_tile_capacity, tiles_per_dim)
        S = decimate(S, r2)
        S, _ = evolve(P, S, r1)
        return S, st, nl
    P = _f32(P)
    S = np.zeros_like(P)
    tpd = np.ascontiguousarray(tiles_per_dim, dtype=np.int64)
    nl = ctypes.c_int64(0)
    st = Stats()
    ns = lib().rdo_ridge_tiled(_fp(P), P.shape[0], P.shape[1], r1, r2, max_tile_capacity,
                               tpd.ctypes.data_as(_I64), _fp(S), ctypes.byref(nl),
                               ctypes.byref(st))
    if ns < 0:
        raise RuntimeError("tile subdivision did not terminate")
    return S[:ns].copy(), st, nl.value


def hausdorff(A, B):
    A, B = _f32(A), _f32(B)
    return lib().rdo_hausdorff(_fp(A), A.shape[0], _fp(B), B.shape[0], A.shape[1])


def evolve_adjoint(P, S0, r1, iters, W):
    P, S0 = _f32(P), _f32(S0)
    W = np.ascontiguousarray(W, dtype=np.float64)
    gP = np.zeros(P.shape, np.float64)
    gS = np.zeros(S0.shape, np.float64)
    Sf = np.zeros_like(S0)
    rc = lib().rdo_evolve_adjoint(_fp(P), P.shape[0], _fp(S0), S0.shape[0], P.shape[1], r1,
                                  iters, W.ctypes.data_as(_D), gP.ctypes.data_as(_D),
                                  gS.ctypes.data_as(_D), _fp(Sf))
    if rc:
        raise MemoryError("oracle adjoint allocation failed")
    return gP, gS, Sf


# --------------------------------------------------------------------------
# reference wrappers (None when oracle/_ref was not built)
# --------------------------------------------------------------------------

class Forward64:
    """FP64 run of the evolve adjoint's forward map with every assignment
    recomputed (rd_fd64.c), kept for central differences of its loss."""

    def __init__(self, P, S0, r1, iters):
        self.P = np.ascontiguousarray(P, dtype=np.float64)
        S0 = np.ascontiguousarray(S0, dtype=np.float64)
        self.np, self.dim = self.P.shape
        self.ns = S0.shape[0]
        self.r1, self.iters = float(r1), int(iters)
        self.S_all = np.zeros((iters + 1, self.ns, self.dim), np.float64)
        self.keys = np.zeros((iters, self.np), np.int32)
        self.cnt = np.zeros((iters, self.ns), np.int32)
        rc = lib().rdo_forward64(self.P.ctypes.data_as(_D), self.np, S0.ctypes.data_as(_D),
                                 self.ns, self.dim, self.r1, self.iters,
                                 self.S_all.ctypes.data_as(_D), self.keys.ctypes.data_as(_I32),
                                 self.cnt.ctypes.data_as(_I32))
        if rc:
            raise MemoryError("rdo_forward64 failed")

    def central_difference(self, W, i, d, h, s0_row=-1):
        """(L(P + h e_id) - L(P - h e_id)) / 2h, L = sum W . S^iters, or None when
        the perturbation changes an assignment.  s0_row: the chosen point that
        starts as a copy of cloud point i (moves with it), or -1."""
        W = np.ascontiguousarray(W, dtype=np.float64)
        out = ctypes.c_double(0.0)
        rc = lib().rdo_fd64(self.P.ctypes.data_as(_D), self.np, self.S_all.ctypes.data_as(_D),
                            self.keys.ctypes.data_as(_I32), self.cnt.ctypes.data_as(_I32),
                            self.ns, self.dim, self.r1, self.iters, W.ctypes.data_as(_D),
                            int(i), int(d), int(s0_row), float(h), ctypes.byref(out))
        if rc == 2:
            raise ValueError("rdo_fd64: bad arguments or allocation failure")
        return None if rc else out.value


def ref_choose(P, r1):
    L = ref()
    P = _f32(P)
    S = np.zeros_like(P)
    ns = L.ref_choose(_fp(P), P.shape[0], P.shape[1], r1, _fp(S))
    return S[:ns].copy()


def ref_evolve_pass(P, S, r1):
    L = ref()
    P, S = _f32(P), _f32(S).copy()
    ns, dim = S.shape
    sums = np.zeros((ns, dim), np.float32)
    cnt = np.zeros(ns, np.int32)
    cont = L.ref_evolve_pass(_fp(P), P.shape[0], _fp(S), ns, dim, r1, _fp(sums),
                             cnt.ctypes.data_as(_I32))
    return S, sums, cnt, cont


def ref_evolve(P, S, r1, threads=0, openmp=False):
    L = ref(openmp)
    P, S = _f32(P), _f32(S).copy()
    L.ref_evolve(_fp(P), P.shape[0], _fp(S), S.shape[0], P.shape[1], r1, threads)
    return S


def ref_evolve_passes_omp(P, S, r1, threads=0, passes=1):
    """`passes` passes of the reference's OpenMP evolve loop body (in place on a
    copy of S); returns (S, cont).  threads=0 uses every core."""
    L = ref(True)
    P, S = _f32(P), _f32(S).copy()
    cont = L.ref_evolve_passes_omp(_fp(P), P.shape[0], _fp(S), S.shape[0], P.shape[1], r1,
                                   threads, passes)
    return S, cont


def ref_decimate(S, r2):
    L = ref()
    S = _f32(S).copy()
    ns = L.ref_decimate(_fp(S), S.shape[0], S.shape[1], r2)
    return S[:ns].copy()


def ref_decimate_nocopy(S, seg_cnt, r2):
    L = ref()
    S = _f32(S).copy()
    seg = np.ascontiguousarray(seg_cnt, dtype=np.int64).copy()
    ns = L.ref_decimate_nocopy(_fp(S), len(seg), seg.ctypes.data_as(_I64), S.shape[1], r2)
    return S[:ns].copy(), seg


def ref_ridge_bf(P, r1, r2, threads=0, openmp=False):
    L = ref(openmp)
    P = _f32(P)
    S = np.zeros_like(P)
    ns = L.ref_bf_ridge(_fp(P), P.shape[0], P.shape[1], r1, r2, _fp(S), threads)
    return S[:ns].copy()


def ref_ridge_tiled(P, r1, r2, max_tile_capacity, tiles_per_dim, threads=1, openmp=False,
                    refine=False):
    L = ref(openmp)
    P = _f32(P)
    S = np.zeros_like(P)
    tpd = np.ascontiguousarray(tiles_per_dim, dtype=np.int64)
    times = np.zeros(4, np.float32)
    ns = L.ref_tiled_ridge(_fp(P), P.shape[0], P.shape[1], r1, r2, max_tile_capacity,
                           tpd.ctypes.data_as(_I64), threads, 1 if refine else 0, _fp(S),
                           _fp(times))
    return S[:ns].copy(), times


def order(S, r2):
    """Greedy chains of order.hpp:45-141: (order, chain_start) int32 arrays."""
    S = _f32(S)
    ns = S.shape[0]
    o = np.empty(max(ns, 1), np.int32)
    cs = np.empty(ns + 1, np.int32)
    nch = lib().rdo_order(_fp(S), ns, S.shape[1], r2,
                          o.ctypes.data_as(_I32), cs.ctypes.data_as(_I32))
    return o[:ns].copy(), cs[:nch + 1].copy()


def ref_order(S, r2):
    """The same chains from the reference's own rd::orderSamples."""
    L = ref(False)
    S = _f32(S)
    ns = S.shape[0]
    o = np.empty(max(ns, 1), np.int32)
    cs = np.empty(ns + 1, np.int32)
    nch = L.ref_order(_fp(S), ns, S.shape[1], r2, o.ctypes.data_as(_I32), cs.ctypes.data_as(_I32))
    return o[:ns].copy(), cs[:nch + 1].copy()


def ref_load_text(path, cap=1 << 22):
    """The reference's own text cloud reader (rd::Samples<float>::loadFromFile).
    It resolves files relative to the running executable's directory, so the
    folder is passed relative to it.  Returns an array, or None when the
    reference throws."""
    L = ref(False)
    exe_dir = os.path.dirname(os.path.realpath("/proc/self/exe"))
    folder = os.path.relpath(os.path.dirname(os.path.abspath(path)), exe_dir) + "/"
    out = np.zeros(cap, np.float32)
    dim = ctypes.c_int(0)
    n = L.ref_load_text(folder.encode(), os.path.basename(path).encode(), _fp(out), cap,
                        ctypes.byref(dim))
    if n < 0:
        return None
    return out[: n * dim.value].reshape(n, dim.value).copy()


def quality(T, I=None, which="hausdorff", use_ref=False):
    """assessment_quality.hpp in float: which = "hausdorff" (T vs ideal I),
    "stats" ((median, avg, min, max) of T's distances to I) or "segment"
    (largest distance of T to the x axis).  use_ref: the reference's own code."""
    L = ref(False) if use_ref else lib()
    pre = "ref_" if use_ref else "rdo_"
    T = _f32(T)
    dim = T.shape[1]
    if which == "segment":
        return getattr(L, pre + "segment_hausdorff_f32")(_fp(T), T.shape[0], dim)
    I = _f32(I)
    if which == "hausdorff":
        return getattr(L, pre + "hausdorff_f32")(_fp(T), T.shape[0], _fp(I), I.shape[0], dim)
    out = np.zeros(4, np.float32)
    getattr(L, pre + "distance_stats_f32")(_fp(T), T.shape[0], _fp(I), I.shape[0], dim, _fp(out))
    return tuple(float(x) for x in out)
