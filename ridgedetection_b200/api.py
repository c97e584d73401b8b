"""Python mirror of the reference's device-facing classes, over the C ABI.

``BruteForceRidgeDetection`` follows rd::gpu::bruteForce::RidgeDetection
(rd/gpu/device/brute_force/simulation.cuh:35-112): construct with
(np, r1, r2), fill the points, call ``ridge_detection()``, then
``get_chosen_samples_count()`` and read the chosen points.

``BatchedRidgeDetection`` solves many independent clouds in one engine run (no
reference counterpart; the reference solves one cloud per call).

Inputs may be numpy arrays (host memory) or CUDA torch tensors (device memory,
enqueued on the current torch stream).  There is no CPU path: everything runs
through librd_b200.so.
"""
from __future__ import annotations

import ctypes
from typing import List, Optional, Sequence, Tuple

import numpy as np

from . import _lib as L

ROW_MAJOR = L.RD_ROW_MAJOR
COL_MAJOR = L.RD_COL_MAJOR
LOOP_GRAPH = L.RD_LOOP_GRAPH
LOOP_HOST = L.RD_LOOP_HOST
TILED_MIXED = 0
TILED_LOCAL = 1


def _is_torch_cuda(x) -> bool:
    return hasattr(x, "is_cuda") and bool(x.is_cuda)


def _ptr_of(x, want_writable=False):
    """(pointer, on_device, stream) of a float32 numpy array or CUDA tensor."""
    if _is_torch_cuda(x):
        import torch
        if x.dtype != torch.float32:
            raise TypeError("points must be float32")
        if not x.is_contiguous():
            raise ValueError("CUDA tensors must be contiguous")
        return ctypes.c_void_p(x.data_ptr()), 1, ctypes.c_void_p(
            torch.cuda.current_stream(x.device).cuda_stream)
    if not isinstance(x, np.ndarray):
        raise TypeError("points must be a numpy array or a CUDA torch tensor")
    if x.dtype != np.float32 or not x.flags["C_CONTIGUOUS"]:
        raise TypeError("numpy points must be C-contiguous float32")
    if want_writable and not x.flags["WRITEABLE"]:
        raise ValueError("output array is read-only")
    return ctypes.c_void_p(x.ctypes.data), 0, ctypes.c_void_p(0)


class BruteForceRidgeDetection:
    """rd::gpu::bruteForce::RidgeDetection<float, DIM, IN_MEM_LAYOUT, OUT_MEM_LAYOUT>."""

    def __init__(self, np_: int, r1: float, r2: float, dim: int,
                 in_layout: int = ROW_MAJOR, out_layout: int = ROW_MAJOR,
                 loop_mode: int = LOOP_GRAPH):
        self._lib = L.lib()
        self._h = ctypes.c_void_p()
        L.check(self._lib.rd_bf_create(ctypes.byref(self._h), dim, in_layout, out_layout,
                                       int(np_), float(r1), float(r2)))
        self.np_ = int(np_)
        self.r1_ = float(r1)
        self.r2_ = float(r2)
        self.dim = int(dim)
        self.in_layout = in_layout
        self.out_layout = out_layout
        self.ns_ = 0
        self.set_loop_mode(loop_mode)

    def set_loop_mode(self, mode: int):
        L.check(self._lib.rd_bf_set_loop_mode(self._h, mode))

    def set_points(self, pts, pitch: int = 0):
        """Copy the cloud into the device (the reference's dP_)."""
        p, dev, st = _ptr_of(pts)
        L.check(self._lib.rd_bf_set_points(self._h, p, int(pitch), dev, st))

    def ridge_detection(self, stream=None):
        st = ctypes.c_void_p(stream) if stream is not None else self._current_stream()
        L.check(self._lib.rd_bf_run(self._h, st))
        self.get_chosen_samples_count()

    def get_chosen_samples_count(self) -> int:
        n = ctypes.c_int64(0)
        L.check(self._lib.rd_bf_get_count(self._h, ctypes.byref(n)))
        self.ns_ = int(n.value)
        return self.ns_

    def chosen_points(self, out=None, pitch: int = 0):
        """Chosen points in the handle's output layout (numpy unless `out` is given)."""
        if out is None:
            if self.out_layout == ROW_MAJOR:
                out = np.empty((self.ns_, self.dim), np.float32)
            else:
                out = np.empty((self.dim, self.ns_), np.float32)
        p, dev, st = _ptr_of(out, want_writable=True)
        L.check(self._lib.rd_bf_get_points(self._h, p, int(pitch), dev, st))
        return out

    def stats(self) -> L.RunStats:
        s = L.RunStats()
        L.check(self._lib.rd_bf_get_stats(self._h, ctypes.byref(s)))
        return s

    @staticmethod
    def _current_stream():
        try:
            import torch
            if torch.cuda.is_available():
                return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
        except Exception:
            pass
        return ctypes.c_void_p(0)

    def close(self):
        if self._h:
            self._lib.rd_bf_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def ridge_detection(P: np.ndarray, r1: float, r2: float, loop_mode: int = LOOP_GRAPH):
    """Brute-force ridge of one ROW_MAJOR float32 cloud; returns (S, stats)."""
    P = np.ascontiguousarray(P, dtype=np.float32)
    rd = BruteForceRidgeDetection(P.shape[0], r1, r2, P.shape[1], loop_mode=loop_mode)
    try:
        rd.set_points(P)
        rd.ridge_detection()
        return rd.chosen_points(), rd.stats()
    finally:
        rd.close()


class TiledRidgeDetection:
    """rd::gpu::tiled::RidgeDetection<DIM, IN, OUT, RD_BRUTE_FORCE, RD_MIXED,
    RD_EXTENDED_TILE, float> (rd/gpu/device/tiled/simulation.cuh:41-241), with the
    results of the reference CPU EXT_TILE_TREE_MIXED_RD implementation."""

    def __init__(self, points_num: int, dim: int, input_points=None,
                 in_layout: int = ROW_MAJOR, out_layout: int = ROW_MAJOR,
                 loop_mode: int = LOOP_GRAPH):
        self._lib = L.lib()
        self._h = ctypes.c_void_p()
        L.check(self._lib.rd_tiled_create(ctypes.byref(self._h), dim, in_layout, out_layout,
                                          int(points_num)))
        self.dim = int(dim)
        self.out_layout = out_layout
        self.ns_ = 0
        L.check(self._lib.rd_tiled_set_loop_mode(self._h, loop_mode))
        if input_points is not None:
            self.set_points(input_points)

    def set_points(self, pts, pitch: int = 0):
        p, dev, st = _ptr_of(pts)
        L.check(self._lib.rd_tiled_set_points(self._h, p, int(pitch), dev, st))

    def __call__(self, r1: float, r2: float, max_tile_capacity: int,
                 tiles_per_dim: Sequence[int], end_phase_refinement: bool = False,
                 stream=None):
        tpd = (ctypes.c_int32 * self.dim)(*[int(t) for t in tiles_per_dim])
        st = ctypes.c_void_p(stream) if stream is not None \
            else BruteForceRidgeDetection._current_stream()
        L.check(self._lib.rd_tiled_run(self._h, float(r1), float(r2), int(max_tile_capacity),
                                       tpd, int(bool(end_phase_refinement)), st))
        return self.get_chosen_points_num()

    ridge_detection = __call__

    def get_chosen_points_num(self) -> int:
        n = ctypes.c_int64(0)
        L.check(self._lib.rd_tiled_get_count(self._h, ctypes.byref(n)))
        self.ns_ = int(n.value)
        return self.ns_

    def get_chosen_points(self, out=None, pitch: int = 0):
        if out is None:
            shape = (self.ns_, self.dim) if self.out_layout == ROW_MAJOR else (self.dim, self.ns_)
            out = np.empty(shape, np.float32)
        p, dev, st = _ptr_of(out, want_writable=True)
        L.check(self._lib.rd_tiled_get_points(self._h, p, int(pitch), dev, st))
        return out

    def get_timers(self):
        v = [ctypes.c_float(0) for _ in range(4)]
        L.check(self._lib.rd_tiled_get_timers(self._h, *[ctypes.byref(x) for x in v]))
        return dict(zip(["whole", "build_tree", "rd_tiles", "refinement"], [x.value for x in v]))

    def leaf_count(self) -> int:
        n = ctypes.c_int64(0)
        L.check(self._lib.rd_tiled_get_leaf_count(self._h, ctypes.byref(n)))
        return int(n.value)

    def set_policy(self, policy: int) -> None:
        """TILED_MIXED (default: global decimation over all leaves) or
        TILED_LOCAL (a complete ridge detection inside every leaf)."""
        L.check(self._lib.rd_tiled_set_policy(self._h, int(policy)))

    def set_profiling(self, enable: bool = True) -> None:
        """Host-loop runs time every fused tile-evolve launch (stats().assign_ms)."""
        L.check(self._lib.rd_tiled_set_profiling(self._h, 1 if enable else 0))

    def stats(self) -> L.RunStats:
        s = L.RunStats()
        L.check(self._lib.rd_tiled_get_stats(self._h, ctypes.byref(s)))
        return s

    def close(self):
        if self._h:
            self._lib.rd_tiled_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def tiled_ridge_detection(P: np.ndarray, r1: float, r2: float, max_tile_capacity: int,
                          tiles_per_dim: Sequence[int], loop_mode: int = LOOP_GRAPH,
                          end_phase_refinement: bool = False, policy: int = TILED_MIXED):
    """Tiled ridge of one ROW_MAJOR float32 cloud; returns (S, stats, n_leaves).
    With end_phase_refinement the result is refined as rd_tiled.hpp:1386-1419
    does (brute-force decimation, then an evolve of the whole cloud)."""
    P = np.ascontiguousarray(P, dtype=np.float32)
    rd = TiledRidgeDetection(P.shape[0], P.shape[1], P, loop_mode=loop_mode)
    try:
        rd.set_policy(policy)
        rd(r1, r2, max_tile_capacity, tiles_per_dim, end_phase_refinement=end_phase_refinement)
        return rd.get_chosen_points(), rd.stats(), rd.leaf_count()
    finally:
        rd.close()


class BatchedRidgeDetection:
    """Many independent clouds, one engine run per point dimension."""

    def __init__(self, loop_mode: int = LOOP_GRAPH):
        self._lib = L.lib()
        self._h = ctypes.c_void_p()
        L.check(self._lib.rd_batch_create(ctypes.byref(self._h)))
        L.check(self._lib.rd_batch_set_loop_mode(self._h, loop_mode))
        self._dims: List[int] = []
        self._counts = np.zeros(0, np.int64)

    def run(self, packed, descs: Sequence[Tuple[int, int, int, float, float]], stream=None):
        """packed: all clouds' ROW_MAJOR floats back to back (numpy or CUDA
        tensor); descs: per cloud (offset_in_floats, n, dim, r1, r2)."""
        arr = (L.CloudDesc * len(descs))()
        for k, (off, n, dim, r1, r2) in enumerate(descs):
            arr[k].offset, arr[k].n, arr[k].dim = int(off), int(n), int(dim)
            arr[k].r1, arr[k].r2 = float(r1), float(r2)
        p, dev, st = _ptr_of(packed)
        if stream is not None:
            st = ctypes.c_void_p(stream)
        total = int(packed.numel() if dev else packed.size)
        L.check(self._lib.rd_batch_run(self._h, arr, len(descs), p, total, dev, st))
        self._dims = [int(d[2]) for d in descs]
        self._counts = np.zeros(len(descs), np.int64)
        L.check(self._lib.rd_batch_get_counts(
            self._h, self._counts.ctypes.data_as(ctypes.POINTER(ctypes.c_int64))))
        return self._counts.copy()

    def chosen_points(self, cloud: int) -> np.ndarray:
        out = np.empty((int(self._counts[cloud]), self._dims[cloud]), np.float32)
        if out.size:
            L.check(self._lib.rd_batch_get_points(self._h, int(cloud),
                                                  ctypes.c_void_p(out.ctypes.data), 0,
                                                  ctypes.c_void_p(0)))
        return out

    def stats(self) -> L.RunStats:
        s = L.RunStats()
        L.check(self._lib.rd_batch_get_stats(self._h, ctypes.byref(s)))
        return s

    def close(self):
        if self._h:
            self._lib.rd_batch_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def pack_clouds(clouds: Sequence[Tuple[np.ndarray, float, float]]):
    """[(P, r1, r2), ...] -> (packed float32 array, descs)."""
    descs, parts, off = [], [], 0
    for P, r1, r2 in clouds:
        P = np.ascontiguousarray(P, dtype=np.float32)
        descs.append((off, P.shape[0], P.shape[1], r1, r2))
        parts.append(P.reshape(-1))
        off += P.size
    packed = np.concatenate(parts) if parts else np.zeros(0, np.float32)
    return np.ascontiguousarray(packed, dtype=np.float32), descs


# ---------------------------------------------------------------------------
# launch-shape tuning (no reference counterpart)
# ---------------------------------------------------------------------------

def tune_set(dim: int, n: int, block: int, items: int, cull_items: int = 4,
             r1: float = 0.0) -> None:
    """Use CTA size ``block`` and ``items`` points per thread for the
    all-pairs assignment (and as the grouping chunk) and ``cull_items`` points
    per lane for the culled assignment, for clouds of dimension ``dim`` whose
    size is in the power-of-two bucket of ``n`` and whose r1 is in the
    half-octave bucket of ``r1`` (r1 <= 0: every radius)."""
    L.check(L.lib().rd_tune_set(dim, n, float(r1), block, items, cull_items))


def tune_get(dim: int, n: int, r1: float = 0.0) -> Tuple[int, int, int]:
    """(block, items, cull_items) the engine will use for a ``dim``-D cloud of
    ``n`` points with radius ``r1``."""
    b, i, c = ctypes.c_int(0), ctypes.c_int(0), ctypes.c_int(0)
    L.check(L.lib().rd_tune_get(dim, n, float(r1), ctypes.byref(b), ctypes.byref(i),
                                ctypes.byref(c)))
    return b.value, i.value, c.value


def tune_reset() -> None:
    """Forget every tuned or set shape (back to the default 128 x 8)."""
    L.check(L.lib().rd_tune_reset())


def set_assign_cull(enable: bool) -> None:
    """Switch the exact chunk-box culling of the brute-force assignment
    (process-wide, on by default).  Results are the same either way; off runs
    the all-pairs assignment kernel."""
    L.check(L.lib().rd_set_assign_cull(1 if enable else 0))


def get_assign_cull() -> bool:
    """Whether runs started now use the culled assignment."""
    e = ctypes.c_int(0)
    L.check(L.lib().rd_get_assign_cull(ctypes.byref(e)))
    return bool(e.value)


def set_tile_clusters(enable: bool, min_points: int = 0, seg_min: int = 0) -> None:
    """Cluster evolve of heavy tiles in tiled runs (changes no result): tiles
    with at least min_points evolve points are evolved by a thread-block
    cluster, keys with at least seg_min members folded in segments across it
    (0 = default threshold).  Process-wide."""
    L.check(L.lib().rd_set_tile_clusters(1 if enable else 0, int(min_points), int(seg_min)))


def get_tile_clusters() -> Tuple[bool, int, int]:
    e, m, s = ctypes.c_int(0), ctypes.c_int64(0), ctypes.c_int64(0)
    L.check(L.lib().rd_get_tile_clusters(ctypes.byref(e), ctypes.byref(m), ctypes.byref(s)))
    return bool(e.value), int(m.value), int(s.value)


def choose_count(P, r1: float) -> int:
    """Number of points the greedy r1-ball choose keeps for the cloud P (a
    float32 CUDA tensor or numpy array, ROW_MAJOR n x dim)."""
    import torch
    dP = P if _is_torch_cuda(P) else torch.from_numpy(np.ascontiguousarray(P, np.float32)).cuda()
    n, dim = dP.shape
    S = torch.empty_like(dP)
    ns = ctypes.c_int64(0)
    stream = torch.cuda.current_stream().cuda_stream
    L.check(L.lib().rd_choose(dim, ctypes.c_void_p(dP.data_ptr()), n, float(r1),
                              ctypes.c_void_p(S.data_ptr()), ctypes.byref(ns),
                              ctypes.c_void_p(stream)))
    return int(ns.value)


def autotune(dim: int, n: int, ns: int, reps: int = 5, points=None,
             r1: float = 2.0) -> Tuple[int, int, int, float]:
    """Time the supported shapes of the assignment in use and keep the best
    (median of five runs, the incumbent kept within 3%) for the (dim, size,
    r1) bucket; returns (block, items, cull_items, microseconds per
    evolve pass).
    With ``points`` (a float32 CUDA tensor, n x dim) the timing runs on that
    cloud with its first ``ns`` points as the chosen set and radius ``r1``;
    otherwise on ``n`` synthetic uniform points."""
    b, i, c, us = ctypes.c_int(0), ctypes.c_int(0), ctypes.c_int(0), ctypes.c_double(0)
    ptr = None
    if points is not None:
        if not _is_torch_cuda(points):
            raise TypeError("points must be a CUDA tensor")
        ptr = ctypes.c_void_p(points.contiguous().data_ptr())
        n = int(points.shape[0])
    L.check(L.lib().rd_autotune(dim, ptr, n, ns, float(r1), reps, ctypes.byref(b),
                                ctypes.byref(i), ctypes.byref(c), ctypes.byref(us), None))
    return b.value, i.value, c.value, us.value


def autotune_solve(dim: int, points, r1: float, r2: float,
                   runs: int = 3) -> Tuple[int, int, int, float]:
    """Time whole brute-force solves (choose to convergence, graph loop) of
    ``points`` (a float32 CUDA tensor, n x dim) with every supported shape of
    the assignment and keep the best for the (dim, size, r1) bucket, with the
    same decision rule as :func:`autotune`; returns (block, items,
    cull_items, milliseconds per solve)."""
    if not _is_torch_cuda(points):
        raise TypeError("points must be a CUDA tensor")
    b, i, c, ms = ctypes.c_int(0), ctypes.c_int(0), ctypes.c_int(0), ctypes.c_double(0)
    pts = points.contiguous()
    L.check(L.lib().rd_autotune_solve(dim, ctypes.c_void_p(pts.data_ptr()), int(pts.shape[0]),
                                      float(r1), float(r2), int(runs), ctypes.byref(b),
                                      ctypes.byref(i), ctypes.byref(c), ctypes.byref(ms), None))
    return b.value, i.value, c.value, ms.value


def order_chains(S, r2: float):
    """Order a ridge into chains (rd::orderSamples, rd/cpu/brute_force/order.hpp:45,
    with the brute-force class's condition: squared distance <= r2*r2).
    S: n x dim float32 points (numpy or CUDA tensor).  Returns (order,
    chain_start) as numpy int32 arrays: the point indices chain by chain,
    each front to back, and the chain offsets (n_chains + 1 entries)."""
    import torch
    dS = S if _is_torch_cuda(S) else torch.from_numpy(np.ascontiguousarray(S, np.float32)).cuda()
    ns = int(dS.shape[0])
    dim = int(dS.shape[1]) if dS.dim() == 2 else 2
    order = torch.empty(max(ns, 1), dtype=torch.int32, device=dS.device)
    starts = torch.empty(ns + 1, dtype=torch.int32, device=dS.device)
    nch = ctypes.c_int64(0)
    stream = torch.cuda.current_stream(dS.device).cuda_stream
    L.check(L.lib().rd_order_chains(dim, ctypes.c_void_p(dS.data_ptr()), ns, float(r2),
                                    ctypes.c_void_p(order.data_ptr()),
                                    ctypes.c_void_p(starts.data_ptr()), ctypes.byref(nch),
                                    ctypes.c_void_p(stream)))
    return order[:ns].cpu().numpy(), starts[: nch.value + 1].cpu().numpy()


# ---------------------------------------------------------------------------
# cloud files in the reference's formats
# ---------------------------------------------------------------------------

def load_text_cloud(path: str) -> np.ndarray:
    """A text cloud as the reference reads it (rd/utils/samples_set.hpp:254-294):
    n = number of newlines, dim counted on the first line (a last value with no
    trailing white space is not counted), one point per non-empty line."""
    n, d = ctypes.c_int64(0), ctypes.c_int(0)
    L.check(L.lib().rd_text_cloud_shape(path.encode(), ctypes.byref(n), ctypes.byref(d)))
    if d.value < 1:
        raise L.RDError(L.RD_ERR_ARG, "no value on the first line")
    out = np.empty((n.value, d.value), np.float32)
    L.check(L.lib().rd_load_text_cloud(path.encode(), ctypes.c_void_p(out.ctypes.data),
                                       n.value, d.value))
    return out


def load_binary_cloud(path: str, n: int, dim: int) -> np.ndarray:
    """n x dim raw ROW_MAJOR float32 values (tests/test_util.hpp:505-551)."""
    out = np.empty((n, dim), np.float32)
    L.check(L.lib().rd_load_binary_cloud(path.encode(), n, dim, ctypes.c_void_p(out.ctypes.data)))
    return out


def save_binary_cloud(path: str, P) -> None:
    """Write P (n x dim float32) as raw ROW_MAJOR floats."""
    P = np.ascontiguousarray(P, np.float32)
    L.check(L.lib().rd_save_binary_cloud(path.encode(), ctypes.c_void_p(P.ctypes.data),
                                         P.shape[0], P.shape[1]))


# ---------------------------------------------------------------------------
# quality of a ridge (rd/utils/assessment_quality.hpp), on the device
# ---------------------------------------------------------------------------

def _dev(x):
    import torch
    if _is_torch_cuda(x):
        return x.contiguous()
    return torch.from_numpy(np.ascontiguousarray(x, np.float32)).cuda()


def hausdorff(T, I) -> float:
    """Symmetric Hausdorff distance of point sets T and I (float, as the
    reference's hausdorffDistance); -1 for an empty T."""
    dT, dI = _dev(T), _dev(I)
    out = ctypes.c_float(0)
    dim = int(dT.shape[1])
    L.check(L.lib().rd_hausdorff(dim, ctypes.c_void_p(dT.data_ptr()), int(dT.shape[0]),
                                 ctypes.c_void_p(dI.data_ptr()), int(dI.shape[0]),
                                 ctypes.byref(out), None))
    return out.value


def distance_stats(S, I) -> Tuple[float, float, float, float]:
    """(median, mean, min, max) of the distances of S's points to the set I
    (setDistanceStats)."""
    dS, dI = _dev(S), _dev(I)
    v = [ctypes.c_float(0) for _ in range(4)]
    L.check(L.lib().rd_distance_stats(int(dS.shape[1]), ctypes.c_void_p(dS.data_ptr()),
                                      int(dS.shape[0]), ctypes.c_void_p(dI.data_ptr()),
                                      int(dI.shape[0]), *[ctypes.byref(x) for x in v], None))
    return tuple(x.value for x in v)


def segment_hausdorff(T) -> float:
    """Largest distance of T's points to the x axis (RDSegmentAssessmentQuality)."""
    dT = _dev(T)
    out = ctypes.c_float(0)
    L.check(L.lib().rd_segment_hausdorff(int(dT.shape[1]), ctypes.c_void_p(dT.data_ptr()),
                                         int(dT.shape[0]), ctypes.byref(out), None))
    return out.value
