"""B200-native ridge detection (choose / evolve / decimate) over a C ABI.

The compute path is librd_b200.so: hand-written sm_100a CUDA kernels driven by
a C++ host engine (ridgedetection_b200/csrc).  This package is the Python-side
mirror of the reference's interface; it never falls back to a CPU path.
"""
from . import generators  # noqa: F401
from ._lib import RDError, RunStats, lib  # noqa: F401
from .api import (COL_MAJOR, LOOP_GRAPH, LOOP_HOST, ROW_MAJOR, TILED_LOCAL,  # noqa: F401
                  TILED_MIXED,
                  BatchedRidgeDetection, BruteForceRidgeDetection, TiledRidgeDetection,
                  autotune, autotune_solve, choose_count, load_binary_cloud, load_text_cloud, order_chains,
                  pack_clouds, save_binary_cloud, hausdorff, distance_stats, segment_hausdorff, ridge_detection,
                  tiled_ridge_detection, tune_get, tune_reset, tune_set, set_assign_cull,
                  get_assign_cull, set_tile_clusters, get_tile_clusters)

__all__ = ["BruteForceRidgeDetection", "BatchedRidgeDetection", "TiledRidgeDetection",
           "ridge_detection", "tiled_ridge_detection",
           "pack_clouds", "order_chains", "hausdorff", "distance_stats", "segment_hausdorff", "load_text_cloud", "load_binary_cloud", "save_binary_cloud", "autotune", "autotune_solve", "choose_count", "tune_get", "tune_set", "tune_reset", "set_assign_cull", "get_assign_cull", "set_tile_clusters", "get_tile_clusters",
           "ROW_MAJOR", "TILED_MIXED", "TILED_LOCAL", "COL_MAJOR", "LOOP_GRAPH", "LOOP_HOST", "RDError",
           "RunStats", "lib", "generators"]
