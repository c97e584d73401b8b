#!/usr/bin/env python
"""Benchmark of the B200 ridge-detection path (one JSON line on rank 0).

Default workload (N=1): brute-force 3D helix, N = 1,000,000 float32 points,
t~U[0,8pi], p = (cos t, sin t, 0.15 t) + N(0, 0.05^2), r1 = 0.15, r2 = 0.3.
One step = one full ridge solve (choose, then evolve/decimate to convergence)
through the library's C ABI.  The metric is evolve pairs/s: the sum over all
evolve passes of (cloud points x chosen points), divided by the solve time.

At N=1 the same line also carries two sub-objects, each timed by the same
rules (warm-up, L2 flush, CUDA events, clocks, e2e, CPU baseline):
  "tiled"    the tiled 2D spiral, N = 10,000,000, 64 x 64 tiles (full solves),
             with the HBM roofline of the fused per-tile evolve kernel;
  "batched"  4,096 clouds (1k..200k points) solved by one batched graph run,
             against the plain per-cloud loop over the same clouds.
--sub none leaves them out.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]
                  [--workload helix3d_1m|sine2d_20k|batch]

--impl reference times the reference's own OpenMP CPU evolve (compiled from its
sources into oracle/_ref/librdref_omp.so) on the same cloud, one evolve pass per
step, on all host cores.  Under torchrun only rank 0 runs it.

For N > 1 every rank solves its own replica of the workload (the single-cloud
brute-force path does not shard); value = pairs of all ranks / max rank time.
"""
from __future__ import annotations

import argparse
import ctypes
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "evolve pairs/s"
UNIT = "pairs/s"
# DRAM traffic of one assignment launch on the helix3d_1m workload, from one
# ncu capture each (dram__bytes_read.sum + dram__bytes_write.sum):
#   k_assign_cull (culled, the default): 16,034,816 + 0 bytes against 20 B of
#     algorithmic traffic per point (12 B sorted point + 4 B slot read, 4 B key
#     written, the keys staying in L2);
#   k_assign (all pairs): 12,039,936 + 0 bytes, the 1,000,000 points x 12 B
#     read once.
# Applies to helix3d_1m only.
ASSIGN_TRAFFIC_BYTES = {"helix3d_1m": 16_034_816}
ALL_PAIRS_TRAFFIC_BYTES = {"helix3d_1m": 12_039_936}


def parse_args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--workload", default="helix3d_1m",
                    choices=["helix3d_1m", "sine2d_20k", "batch", "spiral2d_10m_tiled",
                             "spiral2d_1m_tiled"])
    ap.add_argument("--clouds", type=int, default=4096, help="batch workload: number of clouds")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--sub", default="tiled,batch",
                    help="default workload at N=1: comma list of sub-workloads measured into "
                         "the same JSON line (tiled, batch) or 'none'")
    ap.add_argument("--assign-cull", default="on", choices=["on", "off"],
                    help="exact chunk-box culling of the brute-force assignment (off = all-pairs kernel)")
    ap.add_argument("--shape", default=None,
                    help="BLOCK,ITEMS[,CULL_ITEMS] of the assignment instead of the autotuner's pick "
                         "(a profiler distorts the tuner's timings)")
    ap.add_argument("--profile-run", action="store_true",
                    help="no timing and no JSON line: after --warmup solves, run --steps "
                         "solves with the host-driven loop so that a profiler sees every "
                         "kernel launch (graph-launched kernels inside a conditional "
                         "node are not profiled)")
    return ap.parse_args()


def workload(name):
    from ridgedetection_b200 import generators as G
    if name == "helix3d_1m":
        return G.helix3d(1_000_000), 0.15, 0.3
    if name == "sine2d_20k":
        return G.sine2d(20_000), 0.3, 0.6
    if name == "spiral2d_10m_tiled":
        return G.spiral2d(10_000_000), 0.2, 0.4
    if name == "spiral2d_1m_tiled":  # small case of the same generator, for profilers
        return G.spiral2d(1_000_000), 0.2, 0.4
    raise ValueError(name)


def run_profile(args):
    """Solves with the host-driven loop for profilers (see --profile-run)."""
    import torch
    import ridgedetection_b200 as rdb
    if args.workload == "batch":
        from ridgedetection_b200 import generators as G
        spec = G.batch_spec(args.clouds)
        clouds = [(G.batch_cloud(n, dim, seed), r1, r2) for (n, dim, r1, r2, seed) in spec]
        packed, descs = rdb.pack_clouds(clouds)
        dpk = torch.from_numpy(packed).cuda()
        b = rdb.BatchedRidgeDetection(loop_mode=rdb.LOOP_HOST)
        for _ in range(args.warmup + args.steps):
            b.run(dpk, descs)
        torch.cuda.synchronize()
        print(json.dumps({"profile_run": "batch", "clouds": args.clouds,
                          "solves": args.warmup + args.steps}))
        return
    P, r1, r2 = workload(args.workload)
    n, dim = P.shape
    dP = torch.from_numpy(P).cuda()
    if args.workload.endswith("_tiled"):
        rd = rdb.TiledRidgeDetection(n, dim, loop_mode=rdb.LOOP_HOST)
        rd.set_points(dP)
        solve = lambda: rd(r1, r2, n + 1, (64, 64))  # noqa: E731
    else:
        if args.shape:
            rdb.tune_set(dim, n, *[int(x) for x in args.shape.split(",")], r1=r1)
        else:
            rdb.autotune(dim, n, max(1, rdb.choose_count(dP, r1)), reps=6, points=dP, r1=r1)
        rd = rdb.BruteForceRidgeDetection(n, r1, r2, dim, loop_mode=rdb.LOOP_HOST)
        rd.set_points(dP)
        solve = rd.ridge_detection
    for _ in range(args.warmup):
        solve()
    for _ in range(args.steps):
        solve()
    torch.cuda.synchronize()
    st = rd.stats()
    print(json.dumps({"profile_run": args.workload, "solves": args.warmup + args.steps,
                      "loop_iters_last": st.loop_iters, "evolve_passes_last": st.evolve_passes}))


class ClockSampler:
    """nvidia-smi clock/throttle samples every 200 ms while running."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        self.p = None

    def start(self):
        try:
            self.p = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.Q}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.p = None

    def stop(self):
        if self.p is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.p.terminate()
        try:
            self.p.wait(timeout=5)
        except Exception:
            self.p.kill()
        self.f.flush()
        self.f.seek(0)
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.f.read().splitlines():
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax.append(float(parts[2]))
            except ValueError:
                continue
            for nm, val in zip(names, parts[5:9]):
                if val.lower() == "active":
                    reasons.add(nm)
        os.unlink(self.f.name)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        busy = [s for s in sm if s > 0.5 * max(sm)] or sm
        return {"sm_mhz": statistics.median(busy), "sm_max_mhz": max(smax),
                "reasons": sorted(reasons), "samples": len(sm)}


def dist_setup(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def cpu_baseline(P, r1, target_s=15.0):
    """The reference's OpenMP evolve on this host's cores: a bounded sample of
    whole evolve passes at the chosen set right after choose."""
    import oracle
    if oracle.ref(True) is None:
        return None
    S0 = oracle.choose(P, r1)
    threads = os.cpu_count() or 1
    t = time.perf_counter()
    oracle.ref_evolve_passes_omp(P, S0, r1, threads=threads, passes=1)
    t1 = time.perf_counter() - t
    passes = int(max(1, min(50, target_s / max(t1, 1e-3))))
    t = time.perf_counter()
    oracle.ref_evolve_passes_omp(P, S0, r1, threads=threads, passes=passes)
    dt = time.perf_counter() - t
    pairs = float(P.shape[0]) * S0.shape[0] * passes
    return {"value": pairs / dt, "unit": UNIT, "cores": threads, "kind": "reference",
            "sample": f"{passes} OpenMP evolve passes (rd::evolve_omp loop body) of the "
                      f"{P.shape[0]}-point cloud at the {S0.shape[0]} chosen points after choose, "
                      f"{dt:.1f} s"}


def run_reference_arm(args, world, rank):
    if rank != 0:
        return
    import oracle
    P, r1, r2 = workload(args.workload)
    if oracle.ref(True) is None:
        print(json.dumps({"impl": "reference",
                          "unavailable": "oracle/_ref/librdref_omp.so was not built"}))
        return
    if args.workload.endswith("_tiled"):
        vals, secs = [], []
        cb = None
        for _ in range(args.warmup + args.steps):
            cb = cpu_baseline_tiled(r1, r2)
            vals.append(cb["value"])
            secs.append(cb["seconds"])
        val = statistics.mean(vals[args.warmup:])
        cb["value"] = val
        print(json.dumps({
            "impl": "reference", "metric": "tiled ridge points/s", "value": val,
            "unit": "points/s", "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": 1e3 * statistics.mean(secs[args.warmup:]), "higher_is_better": True,
            "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": args.workload, "cores": cb["cores"]},
            "cpu_baseline": cb,
            "e2e": {"value": val, "unit": "points/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0},
        }))
        return
    S0 = oracle.choose(P, r1)
    threads = os.cpu_count() or 1
    pairs_step = float(P.shape[0]) * S0.shape[0]
    for _ in range(args.warmup):
        oracle.ref_evolve_passes_omp(P, S0, r1, threads=threads, passes=1)
    t = time.perf_counter()
    for _ in range(args.steps):
        oracle.ref_evolve_passes_omp(P, S0, r1, threads=threads, passes=1)
    dt = time.perf_counter() - t
    val = pairs_step * args.steps / dt
    sample = (f"one OpenMP evolve pass (rd::evolve_omp loop body) per step over the "
              f"{P.shape[0]}-point cloud at the {S0.shape[0]} chosen points after choose")
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": val, "unit": UNIT,
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": dt / args.steps * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": args.workload, "cores": threads},
        "cpu_baseline": {"value": val, "unit": UNIT, "cores": threads, "kind": "reference",
                         "sample": sample},
        "e2e": {"value": val, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }))


def run_b200_bf(args, world, rank, local):
    import torch
    import ridgedetection_b200 as rdb
    from ridgedetection_b200 import _lib as L

    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=300),
                                device_id=dev)
    P, r1, r2 = workload(args.workload)
    n, dim = P.shape
    stream = torch.cuda.current_stream()
    dP = torch.from_numpy(P).to(dev)
    l2_flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)
    # launch shape of the assignment from the project's autotuner: whole solves
    # of this cloud, every supported shape (setup, outside every timed region);
    # --shape fixes it instead
    if args.shape:
        tb, ti, tci = [int(x) for x in args.shape.split(",")] + ([4] if args.shape.count(",") == 1 else [])
        rdb.tune_set(dim, n, tb, ti, tci, r1=r1)
        tune_src, tune_ms = "--shape", None
    else:
        tb, ti, tci, tune_ms = rdb.autotune_solve(dim, dP, r1, r2, runs=3)
        tune_src = "rd_autotune_solve (whole solves timed, median of 3 runs per shape)"
    rd = rdb.BruteForceRidgeDetection(n, r1, r2, dim)
    rd.set_points(dP)

    def barrier():
        torch.cuda.synchronize()
        if world > 1:
            torch.distributed.barrier()
            torch.cuda.synchronize()

    for _ in range(max(3, args.warmup)):
        rd.ridge_detection()
    torch.cuda.synchronize()
    st = rd.stats()
    pairs_step = st.pairs
    iters_step = st.loop_iters

    # ---- timed region: K device-resident solves, L2 flushed between them ----
    clock = ClockSampler(local)
    clock.start()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
          for _ in range(args.steps)]
    barrier()
    for k in range(args.steps):
        l2_flush.zero_()
        ev[k][0].record(stream)
        rd.ridge_detection()
        ev[k][1].record(stream)
    barrier()
    step_ms = [a.elapsed_time(b) for a, b in ev]
    clocks = clock.stop()
    ms = sum(step_ms) / len(step_ms)
    ms_t = torch.tensor([ms], device=dev, dtype=torch.float64)
    if world > 1:
        torch.distributed.all_reduce(ms_t, op=torch.distributed.ReduceOp.MAX)
    ms_max = float(ms_t.item())
    value = world * pairs_step / (ms_max * 1e-3)

    # ---- e2e: host (pinned) buffers through the C ABI, copies inside the timing ----
    hP = torch.from_numpy(P).pin_memory()
    hout = torch.empty((n, dim), dtype=torch.float32).pin_memory()
    e2e_ms = []
    barrier()
    for k in range(args.steps):
        l2_flush.zero_()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        rd.set_points(hP.numpy())
        rd.ridge_detection()
        out = hout[: rd.ns_]
        rd.chosen_points(out.numpy())
        b.record(stream)
        b.synchronize()
        e2e_ms.append(a.elapsed_time(b))
    barrier()
    e2e_t = torch.tensor([sum(e2e_ms) / len(e2e_ms)], device=dev, dtype=torch.float64)
    if world > 1:
        torch.distributed.all_reduce(e2e_t, op=torch.distributed.ReduceOp.MAX)
    e2e_val = world * pairs_step / (float(e2e_t.item()) * 1e-3)
    ns_final = rd.ns_

    # ---- dominant kernel: assign, timed per launch in host-loop solves: the
    # bench's own kernel, then the all-pairs kernel for the FP32 roofline ----
    rd.set_loop_mode(rdb.LOOP_HOST)
    lib = L.lib()
    culled = rdb.get_assign_cull()

    def profiled_solve():
        L.check(lib.rd_bf_set_profiling(rd._h, 1))
        rd.ridge_detection()
        s = rd.stats()
        L.check(lib.rd_bf_set_profiling(rd._h, 0))
        return s

    pst = profiled_solve()
    rdb.set_assign_cull(False)
    ast = profiled_solve()
    rdb.set_assign_cull(culled)
    rd.set_loop_mode(rdb.LOOP_GRAPH)
    flops_per_pair = 3 * dim
    assign_ms_avg = pst.assign_ms / max(1, pst.assign_launches)
    ap_ms_avg = ast.assign_ms / max(1, ast.assign_launches)
    ap_flops_per_launch = ast.pairs * flops_per_pair / max(1, ast.assign_launches)
    ap_tflops = ap_flops_per_launch / (ap_ms_avg * 1e-3) / 1e12
    peak = ctypes.c_double(0)
    L.check(lib.rd_probe_fp32_peak(ctypes.byref(peak), ctypes.c_void_p(stream.cuda_stream)))
    nominal = 148 * 128 * 2 * 1.965e9 / 1e12
    hbm_peak, hbm_src = measured_hbm_gbs()
    # culled kernel: per point a sorted point and its slot read, its key written
    cull_bytes = n * (4 * dim + 4 + 4)
    cull_gbs = cull_bytes / (assign_ms_avg * 1e-3) / 1e9
    all_pairs = {"kernel": "k_assign", "bound": "fp32", "achieved": ap_tflops,
                 "peak": peak.value, "unit": "TFLOP/s", "frac": ap_tflops / peak.value,
                 "peak_source": "measured FMA-chain probe (rd_probe_fp32_peak); "
                                f"nominal {nominal:.1f} TFLOP/s at 1965 MHz",
                 "flops_per_pair": flops_per_pair, "ms_per_launch": ap_ms_avg,
                 "launches": ast.assign_launches,
                 # the exact distance takes 9 separately rounded FP32
                 # operations per pair (no FMA may be used), so the pipe's
                 # ceiling in these units is half the FMA FLOP rate
                 "frac_of_nonfused_peak": ap_tflops / (peak.value / 2),
                 "traffic": ALL_PAIRS_TRAFFIC_BYTES.get(args.workload)}
    if culled:
        roofline = {"bound": "hbm", "kernel": "k_assign_cull", "achieved": cull_gbs,
                    "peak": hbm_peak, "unit": "GB/s", "frac": cull_gbs / hbm_peak,
                    "peak_source": hbm_src, "bytes_per_launch": cull_bytes,
                    "ms_per_launch": assign_ms_avg, "launches": pst.assign_launches,
                    "traffic": ASSIGN_TRAFFIC_BYTES.get(args.workload)}
    else:
        roofline = dict(all_pairs)

    # like-for-like with the CPU baseline: evolve passes from the chosen set
    # right after choose, nothing else
    sw_pairs, sw_s, sw_passes = same_work_gpu(dP, r1)
    if world > 1:
        torch.distributed.barrier()
    rd.close()
    del dP, hP, hout, l2_flush
    subs = {}
    if world == 1 and args.workload == "helix3d_1m" and args.sub != "none":
        wanted = set(args.sub.split(","))
        if "tiled" in wanted:
            subs["tiled"] = run_b200_tiled(args, world, rank, local, embedded=True)
            torch.cuda.empty_cache()
        if "batch" in wanted:
            subs["batched"] = run_b200_batch(args, world, rank, local, embedded=True)
            torch.cuda.empty_cache()
    if rank != 0:
        if world > 1:
            torch.distributed.destroy_process_group()
        return
    cpu = None
    if world == 1 and not args.no_cpu_baseline:
        try:
            cpu = cpu_baseline(P, r1)
        except Exception as e:  # the baseline is reported, never the target
            cpu = {"value": None, "unit": UNIT, "cores": os.cpu_count(), "kind": "reference",
                   "sample": f"failed: {e}"}
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
        "steps": args.steps, "warmup": max(3, args.warmup), "ms_per_step": ms_max,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic",
        "config": {"workload": f"{args.workload}: brute-force full solve, N={n}, dim={dim}, "
                               f"r1={r1}, r2={r2}",
                   "l2": "flushed (256 MiB write) between timed steps",
                   "loop": "CUDA graph WHILE node", "parallelism": f"replicas x{world}",
                   "assign": "culled (exact chunk-box culling)" if culled else "all pairs",
                   "assign_shape": {"block": tb, "items": ti, "cull_items": tci,
                                    "source": tune_src, "tuned_ms_per_solve": tune_ms}},
        "solves_per_s": world * 1e3 / ms_max,
        "pairs_per_step": pairs_step, "loop_iters_per_step": iters_step,
        "ns_final": ns_final,
        "roofline": roofline,
        "all_pairs": all_pairs,
        "e2e": {"value": e2e_val, "unit": UNIT, "h2d_bytes_per_step": int(P.nbytes),
                "d2h_bytes_per_step": int(ns_final * dim * 4)},
        # per loop iteration: assign (culled: with the key histogram), chunk
        # scan (with the key bases), scatter, sum+shift (with the control
        # step), decimate (with the loop condition); per solve about 40 more
        # (reset, choose rounds with their survivor compaction, spatial order)
        "gpu_launches": args.steps * (5 * iters_step + 40),
        "clocks": clocks,
        "cpu_baseline": cpu,
    }
    line["same_work"] = {
        "what": "evolve passes over the whole cloud from the chosen set right after choose "
                "(the CPU baseline's work), rd_evolve_ws with caller scratch, per-pass time from "
                "a (k+1)-pass minus a 1-pass call",
        "gpu_pairs_per_s": sw_pairs / sw_s, "gpu_ms_per_pass": sw_s * 1e3,
        "pairs_per_pass": sw_pairs, "passes": sw_passes,
        "cpu_pairs_per_s": cpu["value"] if cpu else None,
        "gpu_over_cpu": (sw_pairs / sw_s / cpu["value"]) if cpu and cpu.get("value") else None,
    }
    line.update(subs)
    print(json.dumps(line))
    if world > 1:
        torch.distributed.destroy_process_group()


def same_work_gpu(dP, r1, passes=20):
    """Evolve passes over the cloud dP from the chosen set right after choose
    -- the work the CPU baseline times -- through rd_evolve_ws with caller
    scratch.  A (passes+1)-pass call and a 1-pass call are timed with CUDA
    events; their difference per pass removes the call's setup.  Returns
    (pairs per pass, seconds per pass, passes run in the long call)."""
    import torch
    from ridgedetection_b200 import _lib as L
    lib = L.lib()
    n, dim = dP.shape
    st = torch.cuda.current_stream()
    vs = ctypes.c_void_p(st.cuda_stream)
    vp = lambda t: ctypes.c_void_p(t.data_ptr())  # noqa: E731
    dS = torch.empty_like(dP)
    tb = ctypes.c_size_t(0)
    ns = ctypes.c_int64(0)
    L.check(lib.rd_choose_ws(dim, vp(dP), n, 0, 0, r1, None, 0, 0, None, None, ctypes.byref(tb), vs))
    ws = torch.empty(tb.value, dtype=torch.uint8, device=dP.device)
    L.check(lib.rd_choose_ws(dim, vp(dP), n, 0, 0, r1, vp(dS), 0, 0, ctypes.byref(ns), vp(ws),
                             ctypes.byref(tb), vs))
    S0 = dS[: ns.value].clone()
    L.check(lib.rd_evolve_ws(dim, vp(dP), n, 0, 0, None, 0, 0, 0, vp(S0), ns.value, 0, 0, r1, passes + 1,
                             None, None, None, ctypes.byref(tb), vs))
    ws = torch.empty(tb.value, dtype=torch.uint8, device=dP.device)
    times = {}
    ran = ctypes.c_int64(0)
    for k in (1, passes + 1, 1, passes + 1):
        S = S0.clone()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(st)
        L.check(lib.rd_evolve_ws(dim, vp(dP), n, 0, 0, None, 0, 0, 0, vp(S), ns.value, 0, 0, r1, k,
                                 ctypes.byref(ran), None, vp(ws), ctypes.byref(tb), vs))
        b.record(st)
        b.synchronize()
        times[k] = (a.elapsed_time(b), ran.value)   # the second round (warm) is kept
    (t1, p1), (tk, pk) = times[1], times[passes + 1]
    per_pass_s = max(1e-9, (tk - t1) * 1e-3 / max(1, pk - p1))
    return float(n) * ns.value, per_pass_s, pk


def measured_hbm_gbs():
    """HBM copy bandwidth measured on this pool (MEASURED_PEAKS.json), else the
    recipe's fallback."""
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"]), "measured (MEASURED_PEAKS.json hbm_gbs)"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback 6.65 TB/s"


def cpu_baseline_tiled(r1, r2, n_sample=1_000_000):
    """The reference's tiled pipeline (EXT_TILE_TREE_MIXED_RD, OpenMP) on a
    bounded sample: the same spiral generator at n_sample points, 64x64 tiles."""
    import oracle
    from ridgedetection_b200 import generators as G
    if oracle.ref(True) is None:
        return None
    Ps = G.spiral2d(n_sample)
    threads = os.cpu_count() or 1
    t = time.perf_counter()
    oracle.ref_ridge_tiled(Ps, r1, r2, n_sample + 1, (64, 64), threads=threads, openmp=True)
    dt = time.perf_counter() - t
    return {"value": n_sample / dt, "unit": "points/s", "cores": threads, "kind": "reference",
            "seconds": dt,
            "sample": f"one OpenMP tiled solve (EXT_TILE_TREE_MIXED_RD) of a {n_sample}-point "
                      f"spiral from the same generator, 64x64 tiles, {dt:.1f} s"}


def run_b200_tiled(args, world, rank, local, embedded=False):
    """Tiled 10M-point spiral: full solves (device tile build, fused per-tile
    evolve, global decimation) through the C ABI, replicas across ranks.
    embedded: measured as a sub-object of the default line (returned, not
    printed; the caller owns the process group)."""
    import torch
    import ridgedetection_b200 as rdb

    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    if world > 1 and not embedded:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=300), device_id=dev)
    wl = "spiral2d_10m_tiled" if embedded else args.workload
    P, r1, r2 = workload(wl)
    n, dim = P.shape
    tiles = (64, 64)
    stream = torch.cuda.current_stream()
    dP = torch.from_numpy(P).to(dev)
    l2_flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)
    rd = rdb.TiledRidgeDetection(n, dim)
    rd.set_points(dP)

    def barrier():
        torch.cuda.synchronize()
        if world > 1:
            torch.distributed.barrier()
            torch.cuda.synchronize()

    for _ in range(max(3, args.warmup)):
        rd(r1, r2, n + 1, tiles)
    torch.cuda.synchronize()
    st = rd.stats()
    pairs_step, point_passes = st.pairs, st.point_passes

    clock = ClockSampler(local)
    clock.start()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
          for _ in range(args.steps)]
    barrier()
    for k in range(args.steps):
        l2_flush.zero_()
        ev[k][0].record(stream)
        rd(r1, r2, n + 1, tiles)
        ev[k][1].record(stream)
    barrier()
    clocks = clock.stop()
    ms = sum(a.elapsed_time(b) for a, b in ev) / args.steps
    ms_t = torch.tensor([ms], device=dev, dtype=torch.float64)
    if world > 1:
        torch.distributed.all_reduce(ms_t, op=torch.distributed.ReduceOp.MAX)
    ms_max = float(ms_t.item())
    ns_final = rd.ns_

    # e2e: pinned host cloud in, ridge out, both inside the timing
    hP = torch.from_numpy(P).pin_memory()
    hout = torch.empty((n, dim), dtype=torch.float32).pin_memory()
    e2e = []
    barrier()
    for k in range(args.steps):
        l2_flush.zero_()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        rd.set_points(hP.numpy())
        rd(r1, r2, n + 1, tiles)
        rd.get_chosen_points(hout[: rd.ns_].numpy())
        b.record(stream)
        b.synchronize()
        e2e.append(a.elapsed_time(b))
    barrier()
    e2e_t = torch.tensor([sum(e2e) / len(e2e)], device=dev, dtype=torch.float64)
    if world > 1:
        torch.distributed.all_reduce(e2e_t, op=torch.distributed.ReduceOp.MAX)
    e2e_ms = float(e2e_t.item())

    # dominant kernel: the fused per-tile evolve, timed per launch in a
    # host-loop solve.  Algorithmic bytes: every pass of a tile streams its
    # points (own + halo) once, DIM x 4 B each.
    rdp = rdb.TiledRidgeDetection(n, dim, loop_mode=rdb.LOOP_HOST)
    rdp.set_points(dP)
    rdp.set_profiling(True)
    rdp(r1, r2, n + 1, tiles)
    pst = rdp.stats()
    rdp.close()
    launches = max(1, pst.assign_launches)
    kern_ms = pst.assign_ms / launches
    bytes_launch = pst.point_passes * dim * 4 / launches
    achieved = bytes_launch / (kern_ms * 1e-3) / 1e9
    peak, peak_src = measured_hbm_gbs()
    timers = rd.get_timers()
    if world > 1:
        torch.distributed.barrier()
    rd.close()
    if rank != 0:
        if world > 1 and not embedded:
            torch.distributed.destroy_process_group()
        return None
    cpu = None
    if world == 1 and not args.no_cpu_baseline:
        try:
            cpu = cpu_baseline_tiled(r1, r2)
        except Exception as e:  # the baseline is reported, never the target
            cpu = {"value": None, "unit": "points/s", "cores": os.cpu_count(),
                   "kind": "reference", "sample": f"failed: {e}"}
    line = {
        "metric": "tiled ridge points/s", "value": world * n / (ms_max * 1e-3),
        "unit": "points/s", "n_gpus": world, "steps": args.steps,
        "warmup": max(3, args.warmup), "ms_per_step": ms_max, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": f"{wl}: tiled (extended tiles, mixed) full solve, "
                               f"N={n}, dim={dim}, r1={r1}, r2={r2}, 64x64 tiles, "
                               f"max tile capacity N+1",
                   "l2": "flushed (256 MiB write) between timed steps",
                   "loop": "CUDA graph WHILE node", "parallelism": f"replicas x{world}"},
        "solves_per_s": world * 1e3 / ms_max,
        "evolve_pairs_per_s": world * pairs_step / (ms_max * 1e-3),
        "pairs_per_step": pairs_step, "ns_final": ns_final,
        "timers_ms": timers,
        # the global decimation: its passes are resolved in parallel rounds
        # (per solve, from the profiling solve)
        "decimation": {"passes": int(pst.dec_passes), "rounds": int(pst.dec_rounds),
                       "rounds_per_pass": pst.dec_rounds / max(1, pst.dec_passes)},
        "roofline": {"bound": "hbm", "kernel": "k_tile_evolve", "achieved": achieved,
                     "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "peak_source": peak_src,
                     "bytes_per_launch": bytes_launch, "kernel_ms_per_launch": kern_ms,
                     "launches": pst.assign_launches, "traffic": None},
        "e2e": {"value": world * n / (e2e_ms * 1e-3), "unit": "points/s",
                "h2d_bytes_per_step": int(P.nbytes), "d2h_bytes_per_step": int(ns_final * dim * 4)},
        # per loop iteration: tile evolve, seven neighbour-list kernels of the
        # global decimation, decimate (with the loop condition); per solve
        # about 12 more (tile build, reset, choose)
        "gpu_launches": args.steps * (12 + 9 * max(1, st.loop_iters)),
        "clocks": clocks,
        "cpu_baseline": cpu,
    }
    if embedded:
        return line
    print(json.dumps(line))
    if world > 1:
        torch.distributed.destroy_process_group()
    return None


def _ref_solve_cloud(item):
    """One cloud of the batch through the reference's serial brute-force
    solve (a worker of cpu_baseline_batch's spawn pool)."""
    import oracle
    from ridgedetection_b200 import generators as G
    n, dim, r1, r2, seed = item
    P = G.batch_cloud(n, dim, seed)
    t = time.perf_counter()
    oracle.ref_ridge_bf(P, r1, r2)
    return time.perf_counter() - t


def cpu_baseline_batch(spec, count=32):
    """The reference has no batched path; its per-cloud CPU solve
    (rd::RidgeDetection<float>, serial build) runs over a bounded sample of the
    batch -- every (len(spec)/count)-th cloud in order of size, so the sample
    spans the size range -- with one cloud per host core at a time (a spawn
    process pool), and the batch's solves/s is extrapolated from it."""
    import multiprocessing as mp
    import oracle
    if oracle.ref() is None:
        return None
    order = sorted(range(len(spec)), key=lambda c: (spec[c][0], c))
    step = max(1, len(spec) // count)
    pick = [spec[order[len(order) - 1 - k * step]] for k in range(min(count, len(spec)))]
    threads = os.cpu_count() or 1
    t = time.perf_counter()
    with mp.get_context("spawn").Pool(threads) as pool:
        secs = pool.map(_ref_solve_cloud, pick, chunksize=1)
    dt = time.perf_counter() - t
    # the whole batch keeps every core busy (thousands of clouds over a few
    # dozen cores), so its rate is the sample's clouds per core-second times
    # the cores; the sample's own wall time is set by its largest cloud
    core_s = sum(secs)
    return {"value": len(pick) * threads / core_s, "unit": "solves/s", "cores": threads,
            "kind": "reference",
            "sample": f"{len(pick)} of the {len(spec)} clouds (every {step}th by size, "
                      f"{min(p[0] for p in pick)}..{max(p[0] for p in pick)} points), each "
                      f"solved by the reference's serial CPU ridge detection, {threads} at a "
                      f"time in a process pool: {core_s:.1f} core-s ({dt:.1f} s wall); "
                      f"solves/s = clouds x cores / core-s"}


def run_b200_batch(args, world, rank, local, embedded=False):
    """Batched workload: graph-driven batched solve vs the plain per-cloud loop.
    Clouds are sharded over ranks by size (LPT, no collective on the data path).
    embedded: measured as a sub-object of the default line (returned, not
    printed; the caller owns the process group)."""
    import torch
    import ridgedetection_b200 as rdb
    from ridgedetection_b200 import generators as G
    from ridgedetection_b200.distributed import shard_lpt

    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    if world > 1 and not embedded:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=600), device_id=dev)
    spec = G.batch_spec(args.clouds)
    mine = [spec[i] for i in shard_lpt([s[0] for s in spec], world)[rank]]
    clouds = [(G.batch_cloud(n, dim, seed), r1, r2) for (n, dim, r1, r2, seed) in mine]
    packed, descs = rdb.pack_clouds(clouds)
    stream = torch.cuda.current_stream()
    dpk = torch.from_numpy(packed).to(dev)
    l2_flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)
    b = rdb.BatchedRidgeDetection()

    def barrier():
        torch.cuda.synchronize()
        if world > 1:
            torch.distributed.barrier()
            torch.cuda.synchronize()

    def max_over_ranks(x):
        t = torch.tensor([x], device=dev, dtype=torch.float64)
        if world > 1:
            torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        return float(t.item())

    for _ in range(max(3, args.warmup)):
        b.run(dpk, descs)
    barrier()
    clock = ClockSampler(local)
    clock.start()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
          for _ in range(args.steps)]
    for k in range(args.steps):
        l2_flush.zero_()
        ev[k][0].record(stream)
        b.run(dpk, descs)
        ev[k][1].record(stream)
    barrier()
    clocks = clock.stop()
    ms_batch = max_over_ranks(sum(a.elapsed_time(c) for a, c in ev) / args.steps)
    stb = b.stats()
    # end to end: pinned packed clouds in, every ridge out, inside the timing
    hpk = torch.from_numpy(packed).pin_memory()
    e2e = []
    for k in range(args.steps):
        a, c = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        dpk.copy_(hpk, non_blocking=True)
        b.run(dpk, descs)
        outs = [b.chosen_points(ci) for ci in range(len(descs))]
        c.record(stream)
        c.synchronize()
        e2e.append(a.elapsed_time(c))
    ms_e2e = max_over_ranks(sum(e2e) / len(e2e))
    d2h = int(sum(o.nbytes for o in outs))
    # plain per-cloud loop: one brute-force handle per cloud, host-synchronised
    # loop (the reference's per-cloud style)
    barrier()
    p0, p1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    p0.record(stream)
    for (P, r1, r2) in clouds:
        rd = rdb.BruteForceRidgeDetection(P.shape[0], r1, r2, P.shape[1],
                                          loop_mode=rdb.LOOP_HOST)
        rd.set_points(torch.from_numpy(P).to(dev))
        rd.ridge_detection()
        rd.close()
    p1.record(stream)
    p1.synchronize()
    ms_plain = max_over_ranks(p0.elapsed_time(p1))
    line = None
    if rank == 0:
        n_all = len(spec)
        cpu = None
        if world == 1 and not args.no_cpu_baseline:
            try:
                cpu = cpu_baseline_batch(spec)
            except Exception as e:  # the baseline is reported, never the target
                cpu = {"value": None, "unit": "solves/s", "cores": os.cpu_count(),
                       "kind": "reference", "sample": f"failed: {e}"}
        line = {
            "metric": "ridge solves/s", "value": n_all / (ms_batch * 1e-3),
            "unit": "solves/s", "n_gpus": world, "steps": args.steps,
            "warmup": max(3, args.warmup), "ms_per_step": ms_batch, "higher_is_better": True,
            "scaling": "strong", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": f"batch of {n_all} clouds (log-uniform 1e3..2e5 points, "
                                   f"half sine2d half helix3d, r1~U[0.1,0.3], r2=2 r1)",
                       "l2": "flushed (256 MiB write) between timed steps",
                       "loop": "CUDA graph WHILE node", "parallelism": f"LPT cloud shards x{world}"},
            "plain_loop_solves_per_s": n_all / (ms_plain * 1e-3),
            "plain_loop_ms": ms_plain,
            "batched_over_plain": ms_plain / ms_batch,
            "pairs_per_step_rank0": stb.pairs, "loop_iters_rank0": stb.loop_iters,
            "e2e": {"value": n_all / (ms_e2e * 1e-3), "unit": "solves/s",
                    "h2d_bytes_per_step": int(packed.nbytes), "d2h_bytes_per_step": d2h},
            # per loop iteration: assign (culled: with the key histogram), two
            # chunk scans (with the key bases), scatter, sum+shift (with the
            # control step), decimate (with the loop condition); per run about
            # 32 more (reset, choose, spatial order)
            "gpu_launches": args.steps * (6 * stb.loop_iters + 32),
            "clocks": clocks,
            "cpu_baseline": cpu,
        }
        if not embedded:
            print(json.dumps(line))
    b.close()
    if world > 1 and not embedded:
        torch.distributed.destroy_process_group()
    return line


def main():
    args = parse_args()
    world, rank, local = dist_setup(args)
    if args.impl != "reference":
        import ridgedetection_b200 as rdb
        rdb.set_assign_cull(args.assign_cull == "on")
    if args.profile_run:
        run_profile(args)
        return
    if args.impl == "reference":
        run_reference_arm(args, world, rank)
        return
    if args.workload == "batch":
        run_b200_batch(args, world, rank, local)
    elif args.workload.endswith("_tiled"):
        run_b200_tiled(args, world, rank, local)
    else:
        run_b200_bf(args, world, rank, local)


if __name__ == "__main__":
    main()
