/*
 * rd_c_api.h -- C ABI of the B200 ridge-detection library (librd_b200.so).
 *
 * Plain pointers and sizes only.  Every call returns an rd_status; nothing
 * exits or traps.  rd_last_error() gives the calling thread's last message.
 * Streams are passed as void* (a cudaStream_t; NULL = legacy default stream).
 * Handles are not thread-safe; distinct handles may be used concurrently.
 *
 * The entry points replace the reference's device-facing interfaces (paths are
 * inside ridge_detection/ of aosewski/RidgeDetection):
 *   rd_bf_*     rd::gpu::bruteForce::RidgeDetection<T,DIM,IN,OUT>
 *               rd/gpu/device/brute_force/simulation.cuh:35-112, .inl:40-434
 *   rd_tiled_*  rd::gpu::tiled::RidgeDetection<DIM,IN,OUT,RD_BRUTE_FORCE,RD_MIXED,
 *               RD_EXTENDED_TILE,T>   rd/gpu/device/tiled/simulation.cuh:41-241
 *   rd_batch_*  no reference counterpart (the reference solves one cloud per call)
 *   rd_evolve_adjoint  no reference counterpart
 *
 * Point layouts follow rd::DataMemoryLayout (rd/utils/memory.h:21-26):
 *   RD_ROW_MAJOR  point i, coordinate d at  p[i * pitch + d]   (pitch >= dim)
 *   RD_COL_MAJOR  point i, coordinate d at  p[d * pitch + i]   (pitch >= n)
 * A pitch of 0 means "packed" (dim for ROW_MAJOR, n for COL_MAJOR).
 * All coordinates are float32.
 */
#ifndef RD_C_API_H
#define RD_C_API_H

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define RD_API __attribute__((visibility("default")))
#else
#define RD_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

typedef enum rd_status {
    RD_OK = 0,
    RD_ERR_ARG = 1,             /* invalid argument                                   */
    RD_ERR_CUDA = 2,            /* a CUDA runtime call failed                          */
    RD_ERR_CAPACITY = 3,        /* a device buffer would overflow                      */
    RD_ERR_NOT_CONVERGED = 4,   /* an iteration limit was reached (results partial)    */
    RD_ERR_ALLOC = 5,           /* device or host allocation failed                    */
    RD_ERR_UNSUPPORTED = 6      /* dimension / option not built into this library      */
} rd_status;

typedef enum rd_layout { RD_ROW_MAJOR = 0, RD_COL_MAJOR = 1 } rd_layout;

/* how the evolve -> decimate -> convergence loop is driven */
typedef enum rd_loop_mode {
    RD_LOOP_GRAPH = 0,  /* CUDA graph with a device-side WHILE node; no host sync per iteration */
    RD_LOOP_HOST = 1    /* host reads a device flag after every iteration (reference style)    */
} rd_loop_mode;

typedef struct rd_run_stats {
    int64_t loop_iters;     /* loop iterations (evolve passes of the slowest cloud)  */
    int64_t evolve_passes;  /* evolve passes summed over clouds                      */
    int64_t max_passes;     /* evolve passes of the cloud that needed most           */
    double  pairs;          /* sum over passes of (cloud points x chosen points)     */
    int32_t err_bits;       /* device error bits (0 when clean)                      */
    int32_t pad;
    double  assign_ms;      /* profiling runs only: summed assign-kernel time (ms)   */
    int64_t assign_launches;/* profiling runs only: assign-kernel launches timed     */
    double  point_passes;   /* sum over clouds of (points x evolve passes): point   */
                            /* coordinates the assignment streams, in points        */
    int64_t dec_passes;     /* decimation passes resolved in parallel rounds         */
    int64_t dec_rounds;     /* rounds those passes took                              */
} rd_run_stats;

RD_API const char* rd_last_error(void);
RD_API int rd_abi_version(void);
/* dimensions compiled into the kernels, as a bit mask (bit d set = dim d) */
RD_API int rd_supported_dims(void);
/* Measurement helper (no reference counterpart): FP32 FMA throughput of the
 * current device from an independent-chain FMA kernel timed with CUDA events,
 * in TFLOP/s (2 flops per FMA).  Used as the FP32 roofline denominator. */
RD_API rd_status rd_probe_fp32_peak(double* tflops, void* stream);
/* Launch-shape tuning (no reference counterpart: the reference's launch
 * shapes are compile-time constants).  When an engine is set up, the
 * assignment's shape is looked up for (dim, floor(log2(points of the largest
 * cloud)), floor(2 log2(r1 of that cloud))): CTA size `block` and points per
 * thread `items` of the all-pairs kernel (block x items is also the chunk of
 * points the grouping kernels work on), and `cull_items`, the points per lane
 * of the culled kernel (a warp's culling box holds 32 x cull_items points of
 * the spatial order).  Supported: block 128 with items 4, 8 or 16, block 256
 * with items 4 or 8; cull_items 2, 4 or 8.  r1 <= 0 stores or looks up an
 * entry valid for every radius.  A lookup takes the exact bucket, else the
 * any-radius entry, else the nearest radius bucket of the same dim and size,
 * else 128 x 8 with cull_items 4.  The table is process-wide and thread-safe;
 * shapes change speed only, never results. */
RD_API rd_status rd_tune_set(int dim, int64_t n, float r1, int block, int items, int cull_items);
RD_API rd_status rd_tune_get(int dim, int64_t n, float r1, int* block, int* items,
                             int* cull_items);
RD_API rd_status rd_tune_reset(void);
/* Exact culling of the brute-force assignment (no reference counterpart; it
 * replaces nothing and changes no result).  rd/cpu/brute_force/evolve.hpp:43-66
 * compares every cloud point with every chosen point but keeps the nearest
 * only when it lies within r1.  With culling on (the default), each chunk of
 * spatially sorted points compares only the chosen points whose distance to
 * the chunk's bounding box can be within r1 (with a rounding margin), giving
 * the same assignment bit for bit.  Off = the all-pairs kernel.  Process-wide,
 * read when a run starts. */
RD_API rd_status rd_set_assign_cull(int enable);
RD_API rd_status rd_get_assign_cull(int* enable);
/* Cluster evolve of heavy tiles (no reference counterpart; it replaces nothing
 * and changes no result).  In tiled runs, a tile with at least min_points
 * evolve points (own + halo) is evolved by a thread-block cluster of 8 CTAs
 * instead of one CTA, and each of its keys with at least seg_min members is
 * folded in 64 warp segments (8 per CTA) whose exact FP32 sums are composed
 * in index order.
 * enable = 0: one CTA per tile.  0 for a threshold keeps its default (100,000
 * points, 8,192 members).  Process-wide, read when a run starts. */
RD_API rd_status rd_set_tile_clusters(int enable, int64_t min_points, int64_t seg_min);
RD_API rd_status rd_get_tile_clusters(int* enable, int64_t* min_points, int64_t* seg_min);
/* Times the supported shapes of the assignment the run would use (culled or
 * all pairs, rd_get_assign_cull) on the cloud d_P (device, n x dim ROW_MAJOR;
 * NULL = n synthetic points uniform in the unit cube) with its first ns points
 * as the chosen set and radius r1: CUDA events around each of `reps` evolve
 * passes (the shape sets the assignment's launch and the chunking of the
 * grouping that follows it; the run's one-time setup is left out); five runs
 * per shape, interleaved over the shapes; the shape with the lowest median
 * time per pass wins, shapes within 2% of it counting as tied (the first of
 * them in the supported order is taken) -- unless the table already holds a
 * shape for this (dim, n, r1) bucket that is within 3% of it, which is kept.  Stores the pick for
 * the bucket and returns it with its median time per pass in microseconds.
 * Runs on `stream` and waits for it; d_P is not modified. */
RD_API rd_status rd_autotune(int dim, const float* d_P, int64_t n, int64_t ns, float r1, int reps,
                             int* block, int* items, int* cull_items, double* us_per_pass,
                             void* stream);
/* The same choice from whole solves: every supported shape solves the cloud
 * d_P (device, n x dim ROW_MAJOR) with radii r1 and r2 from choose to
 * convergence in the CUDA-graph loop, timed with CUDA events, `runs` times
 * (interleaved over the shapes) after one untimed solve each.  The same
 * decision rule as rd_autotune; stores the pick for the (dim, n, r1) bucket
 * and returns it with its median time per solve in milliseconds.  Holds one
 * engine per shape while it runs.  Runs on `stream` and waits for it; d_P is
 * not modified. */
RD_API rd_status rd_autotune_solve(int dim, const float* d_P, int64_t n, float r1, float r2, int runs,
                                   int* block, int* items, int* cull_items, double* ms_per_solve,
                                   void* stream);

/* Orders a ridge into chains: rd::orderSamples (rd/cpu/brute_force/order.hpp:45)
 * with the condition of the brute-force class's order_ option
 * (ridge_detection.inl:148-168), squared distance <= r2*r2.  Every remaining
 * point, in index order, seeds a chain that then takes the first later
 * remaining point within r2 of its front (tested first) or back, until none
 * is left.  d_S: ns x dim ROW_MAJOR device points.  d_order (ns ints)
 * receives the point indices chain by chain, each chain front to back;
 * d_chain_start (ns + 1 ints) the offset of every chain plus the total; the
 * chain count goes to *n_chains (host).  Identical to the reference's chains.
 * Runs on `stream` and waits for it. */
RD_API rd_status rd_order_chains(int dim, const float* d_S, int64_t ns, float r2, int32_t* d_order,
                                 int32_t* d_chain_start, int64_t* n_chains, void* stream);

/* Quality of a ridge (rd/utils/assessment_quality.hpp), on the device, with the
 * reference's float arithmetic; points ROW_MAJOR on the device, results to
 * host floats.  The reference builds its ideal patterns from unseeded random
 * draws, so here the caller passes the ideal set.
 *   rd_hausdorff: max(max over T of dist(t, I), max over I of dist(i, T)),
 *     dist(p, X) = sqrt(min over X of the squared distance); -1 for nt = 0
 *     (hausdorffDistance, :91-121).
 *   rd_distance_stats: median (sorted[n/2]), mean (float sum in sorted order
 *     / n), min and max of dist(s, I) over S (setDistanceStats, :123-154).
 *   rd_segment_hausdorff: the largest distance of a T point to the x axis,
 *     sqrt(sum over d >= 1 of t_d^2); -1 for nt = 0 (RDSegmentAssessmentQuality).
 * Each runs on `stream` and waits for it. */
RD_API rd_status rd_hausdorff(int dim, const float* d_T, int64_t nt, const float* d_I, int64_t ni,
                              float* out, void* stream);
RD_API rd_status rd_distance_stats(int dim, const float* d_S, int64_t n, const float* d_I,
                                   int64_t ni, float* median, float* mean, float* min_dist,
                                   float* max_dist, void* stream);
RD_API rd_status rd_segment_hausdorff(int dim, const float* d_T, int64_t nt, float* out,
                                      void* stream);

/* Cloud files in the reference's formats (host memory, no GPU needed).
 * Text (rd/utils/samples_set.hpp:254-294, :444-462): one point per line.
 * rd_text_cloud_shape gives the point count -- the number of '\n' in the
 * file -- and the dimension counted on the first line the way the reference
 * counts it (values are extracted until end of input is hit; a value that ends
 * the line without trailing white space is not counted).  rd_load_text_cloud
 * then reads every non-empty line as one point into out (n x dim ROW_MAJOR;
 * extra values ignored, missing ones 0); a count of non-empty lines other than
 * n is an error, as in the reference.
 * Binary (tests/test_util.hpp:505-551): n x dim raw ROW_MAJOR floats; the
 * file may be longer than that, not shorter. */
RD_API rd_status rd_text_cloud_shape(const char* path, int64_t* n, int* dim);
RD_API rd_status rd_load_text_cloud(const char* path, float* out, int64_t n, int dim);
RD_API rd_status rd_load_binary_cloud(const char* path, int64_t n, int dim, float* out);
RD_API rd_status rd_save_binary_cloud(const char* path, const float* pts, int64_t n, int dim);

/* Building block of the evolve step (no reference counterpart; the reference
 * forms the same sums inline, rd/cpu/brute_force/evolve.hpp:71-74): for each
 * coordinate d < dim, out[d] = the left-to-right FP32 sum, starting from 0 with
 * one rounding per term, of d_P[d_idx[i]*dim + d] for i = 0..n-1.  method 0
 * evaluates it as a chain of adds, method 1 with the warp-parallel exact
 * evaluation, method 2 with the CTA-wide exact evaluation in rounds, methods
 * 3 and 4 with the warp-segmented evaluation (speculative segment starts,
 * traces composed exactly; 8 and 32 segments) that the tiled evolve kernels
 * use for large clusters; all are bit-identical to the serial loop.  All pointers are device pointers; d_out
 * holds dim floats.  Runs on `stream` and waits for it. */
RD_API rd_status rd_ordered_sum(int dim, const float* d_P, const int32_t* d_idx, int64_t n,
                                float* d_out, int method, void* stream);

/* ---------------------------------------------------------------------------
 * Brute force, one cloud.  Mirrors rd::gpu::bruteForce::RidgeDetection:
 *   ctor(np, r1, r2)            -> rd_bf_create       (simulation.inl:40-90)
 *   caller fills dP_            -> rd_bf_set_points   (tests/test_rd_gpu_simulation/
 *                                                       brute_force/simulation.cu:188-190)
 *   ridgeDetection()            -> rd_bf_run          (simulation.inl:183-384)
 *   getChosenSamplesCount()     -> rd_bf_get_count    (simulation.inl:172-176)
 *   dS_ (ns_ points)            -> rd_bf_get_points
 * ------------------------------------------------------------------------- */
typedef struct rd_bf rd_bf;
RD_API rd_status rd_bf_create(rd_bf** out, int dim, int in_layout, int out_layout, int64_t np,
                       float r1, float r2);
RD_API rd_status rd_bf_set_points(rd_bf* h, const float* pts, int64_t pitch, int src_on_device,
                           void* stream);
RD_API rd_status rd_bf_set_loop_mode(rd_bf* h, int mode);
RD_API rd_status rd_bf_run(rd_bf* h, void* stream);
RD_API rd_status rd_bf_get_count(rd_bf* h, int64_t* ns);
/* out receives ns points in the handle's out_layout (pitch as above, for n = ns) */
RD_API rd_status rd_bf_get_points(rd_bf* h, float* out, int64_t pitch, int dst_on_device, void* stream);
RD_API rd_status rd_bf_get_stats(rd_bf* h, rd_run_stats* st);
/* enable = 1: host-loop runs time every assign-kernel launch with CUDA events
 * (reported in rd_run_stats.assign_ms / assign_launches) */
RD_API rd_status rd_bf_set_profiling(rd_bf* h, int enable);
RD_API rd_status rd_bf_destroy(rd_bf* h);

/* ---------------------------------------------------------------------------
 * Tiled (extended tiles, mixed policy), one cloud.  Mirrors
 * rd::gpu::tiled::RidgeDetection (rd/gpu/device/tiled/simulation.cuh:41-241):
 *   ctor(pointsNum, hostPoints)  -> rd_tiled_create + rd_tiled_set_points
 *   operator()(r1, r2, maxTileCapacity, tilesPerDim[DIM], endPhaseRefinement)
 *                                -> rd_tiled_run
 *   getChosenPointsNum()         -> rd_tiled_get_count
 *   getChosenPoints(T*)          -> rd_tiled_get_points
 *   getTimers()                  -> rd_tiled_get_timers
 * The result is that of the reference CPU implementation
 * rd::tiled::tiledRidgeDetection<EXT_TILE_TREE_MIXED_RD> (rd/cpu/tiled/rd_tiled.hpp:1217-1374):
 * leaf tiles in pre-order, each tile's chosen points in order.  With
 * end_phase_refinement = 1 that result is then refined as rd_tiled.hpp:1386-1419
 * does: a brute-force decimation of the whole set (r2), then an evolve of the
 * entire cloud against the survivors to convergence (r1); the refinement time
 * is the fourth timer.
 * ------------------------------------------------------------------------- */
typedef struct rd_tiled rd_tiled;
RD_API rd_status rd_tiled_create(rd_tiled** out, int dim, int in_layout, int out_layout,
                                 int64_t np);
RD_API rd_status rd_tiled_set_points(rd_tiled* h, const float* pts, int64_t pitch,
                                     int src_on_device, void* stream);
RD_API rd_status rd_tiled_set_loop_mode(rd_tiled* h, int mode);
/* Tile policy, the reference's template argument RD_MIXED / RD_LOCAL
 * (agent_tiled_ridge_detection.cuh:70-90).  RD_TILED_MIXED (default): evolve
 * inside every leaf, decimate globally over all leaves (results as the CPU
 * EXT_TILE_TREE_MIXED_RD).  RD_TILED_LOCAL: a complete ridge detection inside
 * every leaf -- choose over its own points, then evolve over its own and halo
 * points and brute-force decimation until its count stops changing
 * (:232-331 and dispatch_ridge_detection.cuh) -- with the leaves' results in
 * leaf pre-order; the reference appends them in completion order. */
enum { RD_TILED_MIXED = 0, RD_TILED_LOCAL = 1 };
RD_API rd_status rd_tiled_set_policy(rd_tiled* h, int policy);
RD_API rd_status rd_tiled_run(rd_tiled* h, float r1, float r2, int64_t max_tile_capacity,
                              const int32_t* tiles_per_dim, int end_phase_refinement,
                              void* stream);
RD_API rd_status rd_tiled_get_count(rd_tiled* h, int64_t* ns);
RD_API rd_status rd_tiled_get_points(rd_tiled* h, float* out, int64_t pitch, int dst_on_device,
                                     void* stream);
/* whole, tile build, tile ridge detection, end-phase refinement, in ms
 * (TiledRidgeDetectionTimers, rd/gpu/agent/agent_tiled_ridge_detection.cuh:96-102) */
RD_API rd_status rd_tiled_get_timers(rd_tiled* h, float* whole, float* build, float* rd_tiles,
                                     float* refinement);
RD_API rd_status rd_tiled_get_stats(rd_tiled* h, rd_run_stats* st);
/* enable = 1: host-loop runs time every launch of the fused per-tile evolve
 * kernel with CUDA events (reported in rd_run_stats.assign_ms /
 * assign_launches; no reference counterpart) */
RD_API rd_status rd_tiled_set_profiling(rd_tiled* h, int enable);
RD_API rd_status rd_tiled_get_leaf_count(rd_tiled* h, int64_t* n_leaves);
RD_API rd_status rd_tiled_destroy(rd_tiled* h);

/* ---------------------------------------------------------------------------
 * Batched: many independent clouds solved together (brute force per cloud).
 * Cloud c has n points at pts + offset (ROW_MAJOR, packed, offset counted in
 * floats so clouds of different dims can share one array) and its own dim,
 * r1, r2.  Clouds of different dims are solved in separate sub-batches.
 * ------------------------------------------------------------------------- */
typedef struct rd_cloud_desc {
    int64_t offset;   /* first float of the cloud in pts                          */
    int64_t n;        /* number of points                                         */
    int32_t dim;
    float r1, r2;
    int32_t pad;
} rd_cloud_desc;

typedef struct rd_batch rd_batch;
RD_API rd_status rd_batch_create(rd_batch** out);
RD_API rd_status rd_batch_set_loop_mode(rd_batch* h, int mode);
/* pts: packed ROW_MAJOR floats; total_floats = length of pts in floats */
RD_API rd_status rd_batch_run(rd_batch* h, const rd_cloud_desc* clouds, int32_t n_clouds,
                       const float* pts, int64_t total_floats, int src_on_device, void* stream);
RD_API rd_status rd_batch_get_counts(rd_batch* h, int64_t* ns);  /* n_clouds entries */
RD_API rd_status rd_batch_get_points(rd_batch* h, int32_t cloud, float* out, int dst_on_device,
                              void* stream);                 /* ns[cloud]*dim floats */
RD_API rd_status rd_batch_get_stats(rd_batch* h, rd_run_stats* st);
RD_API rd_status rd_batch_destroy(rd_batch* h);

/* ---------------------------------------------------------------------------
 * Device-level steps on caller-owned device buffers (packed ROW_MAJOR f32),
 * replacing the reference's CUB-style device algorithms:
 *   rd_choose    rd::gpu::DeviceChoose::choose      (rd/gpu/device/device_choose.cuh,
 *                dispatch/dispatch_choose.cuh:41); CPU rd::choose (cpu/brute_force/choose.hpp:37)
 *   rd_evolve    rd::gpu::DeviceEvolve::evolve      (rd/gpu/device/device_evolve.cuh:35-62);
 *                CPU rd::evolve (cpu/brute_force/evolve.hpp:293)
 *   rd_decimate  rd::gpu::DeviceDecimate::decimate  (rd/gpu/device/device_decimate.cuh);
 *                CPU rd::decimate (cpu/brute_force/decimate.hpp:41)
 * Each call blocks until its result is in place.  d_S must hold np (choose) or
 * ns (evolve, decimate) points; counts are returned through host pointers.
 * ------------------------------------------------------------------------- */
RD_API rd_status rd_choose(int dim, const float* d_P, int64_t np, float r1, float* d_S,
                           int64_t* ns_out, void* stream);
RD_API rd_status rd_evolve(int dim, const float* d_P, int64_t np, float* d_S, int64_t ns,
                           float r1, int64_t* passes_out, void* stream);
RD_API rd_status rd_decimate(int dim, float* d_S, int64_t ns, float r2, int64_t* ns_out,
                             void* stream);
/* One evolve pass, the body of the reference's evolve loop
 * (rd/cpu/brute_force/evolve.hpp:313-338: calculateClosestSphereCenter then
 * shiftTowardMassCenter; GPU dispatch_evolve.cuh, one iteration of its
 * contFlag loop): every cloud point is assigned to its nearest chosen point
 * within r1, and each chosen point whose cluster mean moved beyond the
 * reference's threshold takes that mean.  *moved_out (host) = 1 when some
 * chosen point moved (the reference's contFlag), else 0.  d_S is updated in
 * place.  Blocks until the result is in place. */
RD_API rd_status rd_evolve_pass(int dim, const float* d_P, int64_t np, float* d_S, int64_t ns,
                                float r1, int32_t* moved_out, void* stream);

/* ---------------------------------------------------------------------------
 * Device-level steps at the reference's full shape: per-array layouts and
 * strides, the neighbour overload of evolve, and CUB-style temporary storage.
 *   rd_choose_ws    DeviceChoose::choose<DIM,IN,OUT>(d_P, d_S, np, d_ns, r,
 *                   pStride, sStride, stream)  (rd/gpu/device/device_choose.cuh)
 *   rd_evolve_ws    DeviceEvolve::evolve<DIM,IN,OUT>(d_P, d_S, d_cordSums,
 *                   d_cnt, np, ns, r, inPtsStride, chosenPtsStride,
 *                   cordSumsStride, stream)  (rd/gpu/device/device_evolve.cuh:35-62)
 *                   and its neighbour overload (d_N, nn, neighbourPtsStride;
 *                   :70-97): the chosen points evolve over the input points
 *                   followed by the neighbour points, in that index order
 *   rd_decimate_ws  DeviceDecimate::decimate<DIM,OUT>(d_S, d_ns, r, stride,
 *                   stream)  (rd/gpu/device/device_decimate.cuh)
 * Every array has its own layout (RD_ROW_MAJOR / RD_COL_MAJOR) and pitch in
 * floats (0 = packed; for rd_choose_ws's COL_MAJOR output, 0 = np, its
 * capacity).  All point arrays are on the device.
 * Temporary storage, as CUB's algorithms take it: call with d_temp = NULL to
 * get the bytes needed in *temp_bytes (nothing runs), then call again with
 * d_temp pointing to at least that many bytes of device memory, 256-byte
 * aligned.  The second call takes all its scratch from d_temp (the reference's
 * d_cordSums / d_spherePointCount are part of it); a d_temp smaller than the
 * query gives RD_ERR_CAPACITY.  The query depends on the sizes, the dimension
 * and the launch-shape table, not on the data.
 * rd_evolve_ws: max_passes = 0 evolves to convergence (RD_ERR_NOT_CONVERGED if
 * the library's limit of 65,536 passes is reached); max_passes = k > 0 stops
 * after at most k passes (k = 1 is one pass of the reference's loop).
 * *passes_out (optional) = passes run; *moved_out (optional) = 1 when the
 * last pass moved a chosen point (the reference's contFlag), else 0.
 * rd_decimate_ws compacts the survivors, in order, to the front of d_S.
 * Each call blocks until its result is in place.
 * ------------------------------------------------------------------------- */
RD_API rd_status rd_choose_ws(int dim, const float* d_P, int64_t np, int p_layout,
                              int64_t p_pitch, float r1, float* d_S, int s_layout,
                              int64_t s_pitch, int64_t* ns_out, void* d_temp,
                              size_t* temp_bytes, void* stream);
RD_API rd_status rd_evolve_ws(int dim, const float* d_P, int64_t np, int p_layout,
                              int64_t p_pitch, const float* d_N, int64_t nn, int n_layout,
                              int64_t n_pitch, float* d_S, int64_t ns, int s_layout,
                              int64_t s_pitch, float r1, int64_t max_passes,
                              int64_t* passes_out, int32_t* moved_out, void* d_temp,
                              size_t* temp_bytes, void* stream);
RD_API rd_status rd_decimate_ws(int dim, float* d_S, int64_t ns, int s_layout, int64_t s_pitch,
                                float r2, int64_t* ns_out, void* d_temp, size_t* temp_bytes,
                                void* stream);

/* ---------------------------------------------------------------------------
 * rd_decimate_noalloc: the decimation of rd_decimate without any device
 * allocation.  It has no counterpart in the reference.  It exists for callers
 * that cannot call cudaMalloc: hosts that forbid device allocation once they
 * have started (real-time or embedded loops, where an allocation can block or
 * fail under memory pressure) and plugins whose device memory belongs to a
 * framework that gives them no workspace.
 *   - Scratch is one fixed __device__ array of RD_DECIMATE_NOALLOC_SCRATCH_BYTES
 *     (1.5 MiB) inside the library; every GPU that loads the library holds it
 *     until the process exits.  ns above RD_DECIMATE_NOALLOC_MAX_POINTS is
 *     rejected with RD_ERR_CAPACITY (use rd_decimate instead).
 *   - The first call on a device (and the first after a device reset) looks up
 *     the array's device address with that device current; make that first
 *     call before any stream capture.
 *   - All calls share the array: calls whose kernels overlap on the GPU race.
 *     Serialize them (one stream, or events).
 *   - d_S (ns points, packed ROW_MAJOR, device) is decimated in place; the
 *     surviving count is written to the device int *d_ns_out (-1 on an internal
 *     error).  The call is asynchronous on `stream` and performs no host sync.
 * ------------------------------------------------------------------------- */
#define RD_DECIMATE_NOALLOC_MAX_POINTS 32768
#define RD_DECIMATE_NOALLOC_SCRATCH_BYTES (1536 * 1024)
RD_API rd_status rd_decimate_noalloc(int dim, float* d_S, int64_t ns, float r2,
                                     int32_t* d_ns_out, void* stream);

/* ---------------------------------------------------------------------------
 * Evolve adjoint (no reference counterpart; the reference is forward-only).
 * Forward: `iters` evolve passes from S0 (ns chosen points, usually copies of
 * cloud points) with the movement test off: each non-empty cluster's point
 * becomes the FP32 mean (index-order sum / count) of its assigned cloud
 * points; empty clusters keep their point.  Decimation is frozen.
 * Reverse for L = sum_k <W_k, S_final_k> with the assignments frozen, in FP64:
 * grad_P (np x dim) = dL/dP through the cluster means; grad_S0 (ns x dim,
 * optional) = dL/dS0, i.e. what flows through clusters that stayed empty.
 * checkpoint_every = 0 keeps every pass's assignment (iters x np ints);
 * k > 0 stores S every k passes and recomputes assignments per segment.
 * on_device selects device (1) or host (0) pointers for all arrays.
 * ------------------------------------------------------------------------- */
RD_API rd_status rd_evolve_adjoint(int dim, const float* P, int64_t np, const float* S0,
                                   int64_t ns, float r1, int iters, int checkpoint_every,
                                   const double* W, float* S_final, double* grad_P,
                                   double* grad_S0, int on_device, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* RD_C_API_H */
