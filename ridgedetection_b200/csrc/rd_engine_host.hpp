// rd_engine_host.hpp -- host side of the batch engine: device buffers, work
// decomposition, the CUDA-graph WHILE loop and the host-synchronised loop.
#pragma once

#include "rd_engine.cuh"

#include <cstdint>
#include <string>
#include <vector>

namespace rdb {

// Caller-provided device scratch (CUB-style temporary storage).  While an
// arena is installed on the calling thread (ArenaScope), every DevBuf::ensure
// carves its buffer out of it (256-byte aligned, bump allocation) instead of
// calling cudaMalloc, and fails with cudaErrorMemoryAllocation when the arena
// is exhausted.  A measuring arena (base == nullptr) only adds up the sizes;
// the buffers it hands out are placeholders that must not be dereferenced,
// so only size planning runs under it (no kernel, no copy).
struct DevArena {
    char* base = nullptr;   // nullptr: measuring
    size_t cap = 0;
    size_t used = 0;
    uint64_t gen = 0;       // set by ArenaScope; buffers from older arenas are stale
    bool exhausted = false; // a request did not fit
    bool measuring() const { return base == nullptr; }
};
DevArena* current_arena();
struct ArenaScope {
    DevArena* prev;
    explicit ArenaScope(DevArena* a);
    ~ArenaScope();
};

// A device buffer that only grows; reused across runs of one engine.
struct DevBuf {
    void* p = nullptr;
    size_t bytes = 0;
    bool borrowed = false;   // carved from an arena: never freed here
    uint64_t gen = 0;        // arena generation it was carved from
    cudaError_t ensure(size_t want);
    void release();
    ~DevBuf() { release(); }
    template <class T>
    T* as() const { return static_cast<T*>(p); }
};

struct RunStats {
    int64_t loop_iters = 0;       // graph/host loop iterations
    int64_t total_passes = 0;     // sum over clouds of evolve passes
    int64_t max_passes = 0;       // max over clouds
    double pairs = 0;             // sum over clouds of sum over passes of n_all*ns
    int err_bits = 0;
    double assign_ms = 0;         // host-loop runs with profile_assign (profile_pass): time
                                  // of the assign kernels (of whole iterations)
    int64_t assign_launches = 0;
    double point_passes = 0;      // sum over clouds of n_all * evolve passes
    int64_t dec_passes = 0;       // decimation passes resolved in parallel rounds
    int64_t dec_rounds = 0;       // rounds they took
};

// Process-wide tuning table: (dim, size bucket, r1 bucket) -> assignment
// launch shape.  The size bucket of a cloud of n points is floor(log2(n)), the
// r1 bucket floor(2 log2(r1)) (half octaves; TUNE_ANY_R1 = an entry for every
// radius).  A lookup takes the exact bucket, else the any-radius entry, else
// the nearest radius bucket of the same dim and size, else the default.
// Entries come from rd_autotune (measured) or rd_tune_set (given).
// Thread-safe.
constexpr int TUNE_ANY_R1 = -100000;
int tune_bucket(int64_t n);
int tune_r1_bucket(float r1);
TuneParams tune_lookup(int dim, int64_t n, float r1);
bool tune_find_exact(int dim, int64_t n, float r1, TuneParams* out);
void tune_store(int dim, int64_t n, float r1, const TuneParams& tp);
void tune_clear();
// supported launch shapes, in a fixed order (culled = the culled kernel's
// candidates: every chunk shape with every box size)
const std::vector<TuneParams>& tune_candidates(bool culled);
// Process-wide switch of the exact chunk-box culling of the assignment (on by
// default); read by every engine run.  Thread-safe.
void set_assign_cull(bool on);
bool assign_cull_enabled();

class Engine {
public:
    Engine();
    ~Engine();
    Engine(const Engine&) = delete;
    Engine& operator=(const Engine&) = delete;

    // Describe the batch.  Clouds must be given with p_off, n_all, n_own, r1,
    // r2 and group filled in; groups with cloud_begin/n_clouds/nocopy.  The
    // clouds of a group must be contiguous and share r2.
    int setup(int dim, const std::vector<CloudDesc>& clouds, const std::vector<GroupDesc>& groups,
              int64_t total_points);

    float* points() { return bP_.as<float>(); }     // packed ROW_MAJOR evolve points
    int64_t total_points() const { return total_points_; }
    int dim() const { return dim_; }

    enum RunMode {
        RUN_FULL = 0,           // choose -> (evolve -> decimate)* to convergence
        RUN_CHOOSE_ONLY = 1,    // choose only
        RUN_EVOLVE_ONLY = 2,    // evolve the given chosen sets to convergence
        RUN_DECIMATE_ONLY = 3,  // one decimation of the given chosen sets
    };
    // Runs on `st`.  use_graph selects the CUDA-graph WHILE loop; otherwise the
    // host reads the loop flag after each iteration (the reference's style).
    // For RUN_EVOLVE_ONLY / RUN_DECIMATE_ONLY the caller first writes each
    // cloud's chosen points at its s_off in chosen_mut() and their counts into
    // given_ns.  Blocks until the run is complete.
    int run(cudaStream_t st, bool use_graph, int mode = RUN_FULL);
    // Size planning for caller-provided scratch: under a measuring arena,
    // after setup(), adds to the arena every buffer that run(st, *, mode)
    // would take for the chosen counts in given_ns (RUN_CHOOSE_ONLY,
    // RUN_EVOLVE_ONLY or RUN_DECIMATE_ONLY).  Launches nothing.
    int plan_workspace(int mode);
    float* chosen_mut() { return bS_.as<float>(); }
    std::vector<int32_t> given_ns;
    // the adjoint's forward step: assign + ordered mean of one pass, no
    // movement test (rd_adjoint.cu); keys()/counts() then hold that pass
    int adjoint_setup(cudaStream_t st);
    int adjoint_step(cudaStream_t st);
    const int32_t* keys() const { return bKeys_.as<int32_t>(); }
    const int32_t* counts() const { return bCnt_.as<int32_t>(); }

    // results, valid after run(): per-cloud chosen count and device pointer
    const std::vector<int32_t>& ns() const { return h_ns_; }
    const std::vector<CloudDesc>& clouds() const { return h_cl_; }
    const float* chosen() const { return bS_.as<float>(); }
    const RunStats& stats() const { return stats_; }
    const std::vector<int32_t>& cloud_err() const { return h_err_; }

    // limits (the reference has none; these keep every loop bounded)
    int max_passes = 1 << 16;
    int max_outer = 4096;
    int max_iters = 1 << 18;
    TuneParams tune{128, 8};
    bool tune_locked = false;     // keep `tune`; otherwise setup() takes tune_lookup()
    bool profile_assign = false;  // host loop only: time every assign launch with events
    bool profile_pass = false;    // host loop only: time every whole iteration instead
                                  // (into assign_ms / assign_launches)
    bool fuse_tiles = true;       // tiled runs: per-tile evolve kernel (see run())
    bool cull_assign = true;      // lockstep passes: exact chunk-box culling of the assignment
    std::string last_error;

private:
    int finish_setup_after_choose(cudaStream_t st);
    void build_tile_order();
    int collect(cudaStream_t st);
    int flags_ = 0;
    int build_graph(cudaStream_t st);
    EngineView view() const;
    int fail(const char* what, cudaError_t e);

    int dim_ = 0;
    int64_t total_points_ = 0;
    std::vector<CloudDesc> h_cl_;
    std::vector<GroupDesc> h_gr_;
    std::vector<int32_t> h_chunk_cloud_, h_slot_cloud_, h_ns_, h_err_;
    std::vector<int64_t> h_dec_hoff_;
    std::vector<int32_t> h_dec_hbits_;
    int32_t n_chunks_ = 0, n_slots_ = 0, n_kblk_ = 0, n_kblk_warp_ = 0;
    int64_t hist_ints_ = 0;  // entries of the chunk x key histogram
    int chunk_pts_ = 1024;
    int chunk_max_ = 0;
    int sms_ = 148;
    int hist_smem_ = 0, scat_smem_ = 0;
    int assign_grid_ = 0;
    RunStats stats_;

    DevBuf bCl_, bGr_, bChunkCloud_, bSlotCloud_;
    DevBuf bP_, bS_, bKeys_, bGrouped_, bPg_, bHist_, bCnt_, bBase_, bBig_, bNext_, bHash_, bSurv_;
    DevBuf bNs_, bPhase_, bCont_, bPasses_, bTotPasses_, bOuter_, bErr_, bPairs_, bCtr_, bKbDone_;
    DevBuf bActCloud_, bActPre_, bGroupConv_, bReady_, bDnbOff_, bDnb_, bDbig_, bDcpre_;
    int dec_smem_max_ = 0;
    int dec_nb_pp_ = DEC_NB_MIN_PER_POINT;
    bool fused_ = false;
    bool cull_ = false;           // this run assigns with culling
    bool spatial_ok_ = false;     // the batch layout allows the spatial order
    DevBuf bPs_, bSorder_, bSpatialTmp_;
    DevBuf bTileOrder_;
    DevBuf bSel_, bSelTmp_;       // GPU-wide choose: survivor list and its compaction scratch
    std::vector<int32_t> h_tile_order_;
    int n_heavy_ = 0;
    int tile_cl_grid_ = 0;
    int tile_seg_min_ = 1 << 30;
    DevBuf bDx_, bDcell_, bDalive_, bDc1_, bDc2_, bDbstart_, bDitems_, bDecHoff_, bDecHbits_;

    cudaStream_t cap_stream_ = nullptr;
    cudaGraphExec_t exec_ = nullptr;
    cudaGraph_t graph_ = nullptr;
    std::vector<unsigned char> graph_key_;
};

}  // namespace rdb
