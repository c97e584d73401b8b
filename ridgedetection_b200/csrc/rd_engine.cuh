// rd_engine.cuh -- the device-side batch engine shared by every entry point.
//
// One engine run solves a batch of independent "clouds" (see CloudDesc) that
// share the point dimension DIM:
//   choose      one CTA per cloud, greedy r1-separated subset in input order
//               over a hashed uniform grid (exact test, grid only prunes);
//   evolve      passes of  assign -> chunk scan -> key bases -> stable
//               scatter -> ordered sum + shift -> control, over all clouds still
//               evolving; the per-chosen coordinate sums are formed in cloud-point
//               index order, exactly as the reference's serial loop forms them;
//   decimate    one CTA per group with the reference's in-order semantics;
//   loop        a device flag says whether any cloud is unfinished; it drives a
//               CUDA-graph WHILE node (graph mode) or is read by the host (plain).
#pragma once

#include "rd_internal.cuh"

#include <cstddef>
#include <cstdint>
#include <string>
#include <vector>

namespace rdb {

enum : int {
    ENG_EVOLVE_ONLY = 1,   // converged clouds finish without decimation
    ENG_ALWAYS_MOVE = 2,   // adjoint forward: every non-empty cluster moves to its mean
};

// neighbour-list capacity of the decimation, per chosen point: at least
// DEC_NB_MIN_PER_POINT, more while the whole list buffer stays within
// DEC_NB_BUDGET entries (lists that do not fit fall back to walking the hash
// buckets)
constexpr int DEC_NB_MIN_PER_POINT = 32;
constexpr int DEC_NB_MAX_PER_POINT = 4096;
constexpr int64_t DEC_NB_BUDGET = int64_t(1) << 28;
// points whose int16 counts live in the decimation's shared memory (a count
// never exceeds the number of points, so int16 holds it)
constexpr int DEC_SMEM_MAX_POINTS = 32752;
// fused per-tile evolve: chosen points per tile it can hold
constexpr int TILE_NS_MAX = 1024;

// kinds of work list over the evolving clouds (rebuilt by the control step
// after every iteration): assignment chunks; blocks of KBLK chosen points of
// clouds with more than SCAN_ROWS_WARP chunks (CTA-wide histogram scan) and of
// the other clouds (one warp per block); chosen slots
enum : int { ACT_CHUNK = 0, ACT_KBLK = 1, ACT_KBLK_WARP = 2, ACT_SLOT = 3, ACT_KINDS = 4 };
constexpr int SCAN_ROWS_WARP = 64;

enum : int {
    CTR_WORK = 0,      // assignment work ticket
    CTR_ACTIVE = 1,    // unfinished clouds after the last control step
    CTR_ITERS = 2,     // loop iterations run
    CTR_ERR = 3,       // OR of global error bits
    CTR_NACT = 4,      // evolving clouds in the current work lists
    CTR_NREADY = 5,    // groups ready for decimation in this iteration
    CTR_NBIG = 6,      // keys in the big-key list of the current pass
    CTR_TILE_HEAVY = 7,// heavy-tile ticket of the cluster tile kernel
    CTR_SUM_DONE = 8,  // CTAs of k_sum_shift finished (the last one runs the control step)
    CTR_DEC_DONE = 9,  // CTAs of k_decimate finished (the last one sets the loop condition)
    CTR_DEC_PASSES = 10,  // decimation passes resolved in parallel rounds (this run)
    CTR_DEC_ROUNDS = 11,  // rounds they took
    CTR_COUNT = 12,
};

struct EngineView {
    const CloudDesc* cl;
    const GroupDesc* gr;
    const int32_t* chunk_cloud;  // chunk -> cloud
    const int32_t* slot_cloud;   // chosen slot -> cloud
    float* P;                    // packed evolve points, ROW_MAJOR
    float* S;                    // chosen points, ROW_MAJOR, capacity n_own per cloud
    int32_t* keys;               // per point slot: assigned chosen index or -1
    int32_t* perm;               // per point slot: point indices grouped by key, index order
                                 // (tiled kernels)
    float* Pg;                   // per point slot: the points' coordinates grouped by key in
                                 // index order, PadDim floats each (lockstep passes)
    int32_t* hist;               // per cloud: n_chunks x ns_cap key histogram (then its prefix over chunks)
    int32_t* cnt;                // per chosen slot: members in the last pass
    int32_t* base;               // per chosen slot: first slot of its segment of perm
    int32_t* big;                // chosen slots with SUM_BIG_MIN+ members in this pass
    int32_t* kbdone;             // per cloud: key blocks of the chunk scan finished in this pass
    int32_t* hash;               // choose hash heads
    int32_t* next;               // per chosen slot: choose hash chain
    int32_t* ns;                 // per cloud: current chosen count
    int32_t* phase;              // per cloud: PH_*
    int32_t* cont;               // per cloud: a coordinate moved in this pass
    int32_t* passes;             // per cloud: passes of the current evolve run
    int32_t* total_passes;       // per cloud: all passes
    int32_t* outer;              // per cloud: evolve/decimate rounds
    int32_t* err;                // per cloud: ERRB_* bits
    unsigned long long* pairs;   // per cloud: sum over passes of n_all * ns
    int32_t* ctr;                // CTR_* counters
    int32_t* act_cloud;          // evolving clouds, in cloud order (n_clouds)
    int32_t* act_pre;            // ACT_KINDS x (n_clouds+1) exclusive prefixes of their work items
    int32_t* group_conv;         // per group: members converged in this round
    int32_t* ready;              // groups ready for decimation (n_groups)
    // decimation scratch, per group (offsets in GroupDesc / dec_hoff)
    float* dx;                   // coordinates of the group's chosen points
    int32_t* dcell;              // their grid cells
    int32_t* dalive;
    int32_t* dc1;                // alive neighbours within r2 (self included)
    int32_t* dc2;                // alive neighbours within 2*r2 (self included)
    int32_t* dbstart;            // bucket starts (HB+1 per group)
    int32_t* ditems;             // bucket members
    int32_t* dnb_off;            // per group: neighbour-list offsets (total+1)
    int32_t* dnb;                // per group: neighbour lists, dec_nb_pp per scratch slot
    int32_t* dbig;               // GPU-wide prepared decimation: {state, group, total}
    int32_t* dcpre;              // its members' chosen-count prefix (n_clouds+1)
    int32_t dec_smem_max;        // points whose counts fit the decimation's shared memory
    int32_t dec_nb_pp;           // neighbour-list entries per scratch slot
    const int64_t* dec_hoff;     // per group: start of its bucket arrays
    const int32_t* dec_hbits;    // per group: log2 buckets
    int32_t n_clouds;
    int32_t n_groups;
    int32_t n_chunks;
    int32_t n_slots;
    int32_t n_kblk;              // blocks of KBLK chosen slots, clouds of > SCAN_ROWS_WARP chunks
    int32_t n_kblk_warp;         // the same over the other clouds
    int32_t chunk_pts;           // max points per assignment chunk (BLOCK*ITEMS)
    int32_t chunk_max;           // largest chunk actually used (scatter staging)
    int32_t hist_smem;           // ints of dynamic smem for the assign histogram
    int32_t scat_smem;           // ints of dynamic smem per scatter warp
    int32_t max_passes;
    int32_t max_outer;
    int32_t max_iters;
    int32_t n_sms;
    int32_t flags;               // ENG_* run-mode bits
    // exact chunk-box culling of the assignment (see k_assign_cull)
    const float* Ps;             // evolve points in spatial order inside each cloud
    const int32_t* sorder;       // spatial position -> packed point slot
    const int32_t* srow;         // spatial position -> its slot's chunk in the cloud (histogram row)
    int32_t cull;                // passes assign with k_assign_cull + k_keyhist
    // fused tiled runs: tiles by decreasing evolve points, the first n_heavy
    // evolved by whole thread-block clusters (rd_tile_cluster.cuh)
    const int32_t* tile_order;
    int32_t n_heavy;
    int32_t tile_cl_grid;        // CTAs of the cluster tile kernel (0 = one-CTA kernel)
    int32_t tile_seg_min;        // members of a key the cluster folds in segments
};

// dynamic shared memory of the decimation kernel: two int16 counts and an
// alive byte per point, then a candidate bit per point
inline int dec_smem_bytes(const EngineView& v)
{
    return ((v.dec_smem_max * 5 + 15) / 16) * 16 + 4 * ((v.dec_smem_max + 31) / 32) + 16;
}

// launch configuration picked by the tuner per (dim, cloud size, r1) bucket
struct TuneParams {
    int block;          // assign CTA size (all-pairs kernel); with items, the chunk size
    int items;          // points per assign thread
    int cull_items = 4; // culled kernel: points per lane (a warp's box holds 32 x this)
};

// host-side launchers (rd_kernels.cu); all enqueue on `st`
cudaError_t launch_choose(int dim, const EngineView& v, cudaStream_t st);
// The cluster path of fused tiled runs (process-wide, read when a run
// starts): on/off (off = one CTA per tile), the evolve points from which a
// tile is evolved by a whole cluster and the members from which a key is
// folded in segments across it.
struct TileClusterParams {
    bool enabled;
    int min_points;
    int seg_min;
};
TileClusterParams tile_cluster_params();
void set_tile_cluster_params(const TileClusterParams& p);
TileClusterParams tile_cluster_defaults();
// choose of one large cloud c (n own points) in GPU-wide rounds; v.hash must
// hold choose_hash_buckets() ints and surv n bytes
cudaError_t launch_choose_rounds(int dim, const EngineView& v, int c, int n, uint8_t* surv,
                                 int32_t* sel, void* tmp, size_t tmp_bytes, cudaStream_t st);
// scratch of the survivor compaction of launch_choose_rounds for n points;
// sel holds n + 1 ints (the list, then its length)
size_t choose_select_scratch_bytes(int64_t n);
int choose_hash_buckets();
cudaError_t prepare_pass(int dim, const EngineView& v, const TuneParams& tp);
// How an iteration ends: the last CTA of its decimation kernel rebuilds the
// work lists and sets the loop condition (k_loopcond's step), leaving the
// count of unfinished clouds in ctr[CTR_ACTIVE] and, with use_handle, setting
// the graph WHILE handle.
struct LoopCond {
    cudaGraphConditionalHandle h = 0;
    int use_handle = 0;
};
// One iteration: evolve pass, control, decimation, loop condition.  a0/a1
// (optional) are recorded on `st` right before and after the assign kernel.
cudaError_t launch_pass(int dim, const EngineView& v, const TuneParams& tp, int assign_grid,
                        const LoopCond& lc, cudaStream_t st, cudaEvent_t a0 = nullptr,
                        cudaEvent_t a1 = nullptr);
// Sets the loop condition and rebuilds the work lists of the next iteration
// as a kernel of its own (count_iter = 0 for the initial build before the
// first iteration).
cudaError_t launch_loopcond(const EngineView& v, cudaGraphConditionalHandle h, int use_handle,
                            cudaStream_t st, int count_iter = 1);
cudaError_t launch_reset(const EngineView& v, cudaStream_t st);
// phases from the chosen counts already in v.ns (evolve or decimate from a given set)
cudaError_t launch_set_given(const EngineView& v, int queue_decimation, cudaStream_t st);
// fused per-tile evolve (every active cloud to convergence, one CTA each) +
// decimation of the groups that became ready; needs every ns <= TILE_NS_MAX
cudaError_t prepare_tile_pass(int dim, const EngineView& v, int* cl_grid);
// a0/a1 (optional) are recorded right before and after the tile-evolve kernel;
// the iteration ends with the loop condition as in launch_pass
cudaError_t launch_tile_pass(int dim, const EngineView& v, const LoopCond& lc, cudaStream_t st,
                             cudaEvent_t a0 = nullptr, cudaEvent_t a1 = nullptr);
cudaError_t launch_decimate(int dim, const EngineView& v, cudaStream_t st);
// quality metrics (rd_quality.cu)
cudaError_t launch_min_dist(int dim, const float* A, int na, const float* B, int nb, float* out,
                            cudaStream_t st);
cudaError_t launch_axis_dist(int dim, const float* T, int n, float* out, cudaStream_t st);
cudaError_t launch_max2(const float* a, int na, const float* b, int nb, float* out, cudaStream_t st);
cudaError_t launch_dist_stats(float* d, int n, float* sorted, int32_t* iota, void* temp,
                              size_t temp_bytes, float* out, cudaStream_t st);
size_t dist_stats_temp_bytes(int n);
// chains of a ridge (rd_order.cu): alive ns bytes, deq 2*ns+1 ints of scratch;
// order ns ints, chain_start ns+1 ints, n_chains one int (all device)
cudaError_t launch_order_chains(int dim, const float* S, int ns, float rsq, unsigned char* alive,
                                int32_t* deq, int32_t* order, int32_t* chain_start,
                                int32_t* n_chains, cudaStream_t st);
// out[d] = ordered FP32 sum of P[idx[i]*dim + d] (method 0 chain, 1 parallel exact)
cudaError_t launch_ordered_sum(int dim, const float* P, const int32_t* idx, int n, float* out,
                               int method, cudaStream_t st);
// Spatial order of every cloud's points for the culled assignment: cells of
// edge r1/4, Morton order of the cells (cloud first), slot order inside a
// cell; Ps/sorder receive the reordered points and their slots.  Needs
// contiguous clouds in cloud order and n_points < 2^31; scratch of
// spatial_prep_scratch_bytes(n).
size_t spatial_prep_scratch_bytes(int64_t n_points);
cudaError_t launch_spatial_prep(int dim, const EngineView& v, int64_t n_points, void* scratch,
                                size_t scratch_bytes, float* Ps, int32_t* sorder, cudaStream_t st);
// the five kernels of one evolve pass without control/decimation (adjoint forward)
cudaError_t launch_evolve_step(int dim, const EngineView& v, const TuneParams& tp, int assign_grid,
                               cudaStream_t st);
int assign_smem_bytes(int dim, const TuneParams& tp, int hist_ints);
int max_assign_blocks_per_sm(int dim, const TuneParams& tp, int hist_ints);
bool tune_supported(int dim, const TuneParams& tp);

}  // namespace rdb
