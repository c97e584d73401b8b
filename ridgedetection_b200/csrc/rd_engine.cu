// rd_engine.cu -- host side of the batch engine (see rd_engine_host.hpp).
#include "rd_engine_host.hpp"

#include <algorithm>
#include <cmath>
#include <tuple>
#include <atomic>
#include <cstring>
#include <map>
#include <mutex>

namespace rdb {

// ---------------------------------------------------------------------------
// tuning table
// ---------------------------------------------------------------------------
namespace {
std::mutex g_tune_mu;
// (dim, size bucket, r1 bucket) -> shape; r1 bucket TUNE_ANY_R1 = any radius
std::map<std::tuple<int, int, int>, TuneParams> g_tune;
}  // namespace

int tune_bucket(int64_t n)
{
    int b = 0;
    while (b < 62 && (int64_t(1) << (b + 1)) <= std::max<int64_t>(n, 1)) ++b;
    return b;
}

int tune_r1_bucket(float r1)
{
    if (!(r1 > 0.0f) || !(r1 < INFINITY)) return TUNE_ANY_R1;
    const double b = std::floor(2.0 * std::log2((double)r1));   // half octaves
    return (int)std::max(-256.0, std::min(256.0, b));
}

TuneParams tune_lookup(int dim, int64_t n, float r1)
{
    std::lock_guard<std::mutex> lk(g_tune_mu);
    const int nb = tune_bucket(n), rb = tune_r1_bucket(r1);
    auto it = g_tune.find({dim, nb, rb});
    if (it != g_tune.end()) return it->second;
    it = g_tune.find({dim, nb, TUNE_ANY_R1});
    if (it != g_tune.end()) return it->second;
    // the nearest radius bucket tuned for this dimension and size
    const TuneParams* best = nullptr;
    int bd = 1 << 30;
    for (const auto& kv : g_tune) {
        if (std::get<0>(kv.first) != dim || std::get<1>(kv.first) != nb) continue;
        const int d = std::abs(std::get<2>(kv.first) - rb);
        if (d < bd) { bd = d; best = &kv.second; }
    }
    return best ? *best : TuneParams{128, 8, 4};
}

bool tune_find_exact(int dim, int64_t n, float r1, TuneParams* out)
{
    std::lock_guard<std::mutex> lk(g_tune_mu);
    auto it = g_tune.find({dim, tune_bucket(n), tune_r1_bucket(r1)});
    if (it == g_tune.end()) return false;
    *out = it->second;
    return true;
}

void tune_store(int dim, int64_t n, float r1, const TuneParams& tp)
{
    std::lock_guard<std::mutex> lk(g_tune_mu);
    g_tune[{dim, tune_bucket(n), tune_r1_bucket(r1)}] = tp;
}

void tune_clear()
{
    std::lock_guard<std::mutex> lk(g_tune_mu);
    g_tune.clear();
}

const std::vector<TuneParams>& tune_candidates(bool culled)
{
    static const std::vector<TuneParams> all_pairs = {
        {128, 4, 4}, {128, 8, 4}, {128, 16, 4}, {256, 4, 4}, {256, 8, 4}};
    static const std::vector<TuneParams> cull = [] {
        std::vector<TuneParams> c;
        for (const TuneParams& s : all_pairs)
            for (int ci : {2, 4, 8}) c.push_back(TuneParams{s.block, s.items, ci});
        return c;
    }();
    return culled ? cull : all_pairs;
}


static std::atomic<int> g_assign_cull{1};
void set_assign_cull(bool on) { g_assign_cull.store(on ? 1 : 0); }
bool assign_cull_enabled() { return g_assign_cull.load() != 0; }

namespace {
thread_local DevArena* t_arena = nullptr;
std::atomic<uint64_t> g_arena_gen{1};
constexpr size_t ARENA_ALIGN = 256;
}  // namespace

DevArena* current_arena() { return t_arena; }

ArenaScope::ArenaScope(DevArena* a) : prev(t_arena)
{
    a->gen = g_arena_gen.fetch_add(1);
    t_arena = a;
}

ArenaScope::~ArenaScope() { t_arena = prev; }

cudaError_t DevBuf::ensure(size_t want)
{
    if (want == 0) want = 16;
    if (DevArena* a = t_arena) {
        if (borrowed && gen == a->gen && want <= bytes) return cudaSuccess;
        release();
        const size_t off = (a->used + ARENA_ALIGN - 1) / ARENA_ALIGN * ARENA_ALIGN;
        if (!a->measuring() && (off > a->cap || want > a->cap - off)) {
            a->exhausted = true;
            return cudaErrorMemoryAllocation;
        }
        // a measuring arena hands out distinct, aligned placeholders
        p = a->measuring() ? reinterpret_cast<void*>(uintptr_t(ARENA_ALIGN) + off) : a->base + off;
        a->used = off + want;
        bytes = want;
        borrowed = true;
        gen = a->gen;
        return cudaSuccess;
    }
    if (want <= bytes && !borrowed) return cudaSuccess;
    release();
    cudaError_t e = cudaMalloc(&p, want);
    if (e != cudaSuccess) {
        p = nullptr;
        bytes = 0;
        return e;
    }
    bytes = want;
    return cudaSuccess;
}

void DevBuf::release()
{
    if (p && !borrowed) cudaFree(p);
    p = nullptr;
    bytes = 0;
    borrowed = false;
}

Engine::Engine() {}

Engine::~Engine()
{
    if (exec_) cudaGraphExecDestroy(exec_);
    if (graph_) cudaGraphDestroy(graph_);
    if (cap_stream_) cudaStreamDestroy(cap_stream_);
}

int Engine::fail(const char* what, cudaError_t e)
{
    last_error = std::string(what) + ": " + cudaGetErrorString(e);
    return 2;  // RD_ERR_CUDA
}

#define RD_CK(call)                                   \
    do {                                              \
        cudaError_t e_ = (call);                      \
        if (e_ != cudaSuccess) return fail(#call, e_); \
    } while (0)

template <class T>
static cudaError_t upload(DevBuf& b, const std::vector<T>& h, cudaStream_t st)
{
    cudaError_t e = b.ensure(sizeof(T) * (h.size() + 1));
    if (e != cudaSuccess || h.empty()) return e;
    if (DevArena* a = current_arena(); a && a->measuring()) return cudaSuccess;
    return cudaMemcpyAsync(b.p, h.data(), sizeof(T) * h.size(), cudaMemcpyHostToDevice, st);
}

int Engine::setup(int dim, const std::vector<CloudDesc>& clouds,
                  const std::vector<GroupDesc>& groups, int64_t total_points)
{
    if (!dim_supported(dim)) {
        last_error = "dim must be 1 to 4";
        return 6;  // RD_ERR_UNSUPPORTED
    }
    if (!tune_locked) {
        int64_t nmax = 1;
        float r1 = 0.0f;
        for (const CloudDesc& cd : clouds)
            if (cd.n_all >= nmax) {
                nmax = std::max<int64_t>(nmax, cd.n_all);
                r1 = cd.r1;
            }
        tune = tune_lookup(dim, nmax, r1);
    }
    if (!tune_supported(dim, tune)) {
        last_error = "unsupported tuning parameters";
        return 1;
    }
    dim_ = dim;
    total_points_ = total_points;
    h_cl_ = clouds;
    h_gr_ = groups;
    chunk_pts_ = tune.block * tune.items;
    int dev = 0;
    RD_CK(cudaGetDevice(&dev));
    RD_CK(cudaDeviceGetAttribute(&sms_, cudaDevAttrMultiProcessorCount, dev));
    // Chunks split every cloud evenly into at most chunk_pts_ points each.  A
    // cloud big enough to fill the GPU on its own gets a multiple of the SM
    // count, so that the single wave of assignment CTAs is balanced.
    int64_t chunk = 0, s_off = 0;
    chunk_max_ = 0;
    h_chunk_cloud_.clear();
    for (size_t c = 0; c < h_cl_.size(); ++c) {
        CloudDesc& cd = h_cl_[c];
        cd.s_off = s_off;
        s_off += cd.n_own;
        cd.chunk_begin = chunk;
        int64_t nch = (cd.n_all + chunk_pts_ - 1) / chunk_pts_;
        if (h_cl_.size() == 1 && nch >= 2 * sms_) nch = (nch + sms_ - 1) / sms_ * sms_;
        cd.n_chunks = (int32_t)nch;
        if (nch > 0)
            chunk_max_ = std::max<int>(chunk_max_, (int)((cd.n_all + nch - 1) / nch));
        for (int k = 0; k < cd.n_chunks; ++k) h_chunk_cloud_.push_back((int32_t)c);
        chunk += cd.n_chunks;
    }
    n_chunks_ = (int32_t)chunk;
    const size_t nc = h_cl_.size();
    // the spatial order sorts by (cloud, cell): clouds must tile [0, total)
    // in cloud order
    spatial_ok_ = total_points < (int64_t(1) << 31) - 1;
    int64_t next_off = 0;
    for (const CloudDesc& cd : h_cl_) {
        spatial_ok_ = spatial_ok_ && cd.p_off == next_off;
        next_off += cd.n_all;
    }
    spatial_ok_ = spatial_ok_ && next_off == total_points;
    RD_CK(bP_.ensure(sizeof(float) * (size_t)(total_points * dim + 4)));
    RD_CK(bS_.ensure(sizeof(float) * (size_t)(s_off * dim + 4)));
    RD_CK(bNext_.ensure(sizeof(int32_t) * (size_t)(s_off + 1)));
    RD_CK(bKeys_.ensure(sizeof(int32_t) * (size_t)(total_points + 1)));
    RD_CK(bGrouped_.ensure(sizeof(int32_t) * (size_t)(total_points + 4)));
    RD_CK(bPg_.ensure(sizeof(float) * (size_t)(total_points * pad_dim(dim) + 4)));
    RD_CK(bNs_.ensure(4 * (nc + 1)));
    RD_CK(bPhase_.ensure(4 * (nc + 1)));
    RD_CK(bCont_.ensure(4 * (nc + 1)));
    RD_CK(bPasses_.ensure(4 * (nc + 1)));
    RD_CK(bTotPasses_.ensure(4 * (nc + 1)));
    RD_CK(bOuter_.ensure(4 * (nc + 1)));
    RD_CK(bErr_.ensure(4 * (nc + 1)));
    RD_CK(bPairs_.ensure(8 * (nc + 1)));
    RD_CK(bCtr_.ensure(4 * CTR_COUNT));
    RD_CK(bKbDone_.ensure(4 * (nc + 1)));
    RD_CK(bActCloud_.ensure(4 * (nc + 1)));
    RD_CK(bActPre_.ensure(4 * ACT_KINDS * (nc + 1)));
    RD_CK(bGroupConv_.ensure(4 * (h_gr_.size() + 1)));
    RD_CK(bReady_.ensure(4 * (h_gr_.size() + 1)));
    RD_CK(bDbig_.ensure(4 * 4));
    RD_CK(bDcpre_.ensure(4 * (nc + 1)));
    return 0;
}

EngineView Engine::view() const
{
    EngineView v;
    std::memset(&v, 0, sizeof(v));
    v.cl = bCl_.as<CloudDesc>();
    v.gr = bGr_.as<GroupDesc>();
    v.chunk_cloud = bChunkCloud_.as<int32_t>();
    v.slot_cloud = bSlotCloud_.as<int32_t>();
    v.P = bP_.as<float>();
    v.S = bS_.as<float>();
    v.keys = bKeys_.as<int32_t>();
    v.perm = bGrouped_.as<int32_t>();
    v.Pg = bPg_.as<float>();
    v.hist = bHist_.as<int32_t>();
    v.cnt = bCnt_.as<int32_t>();
    v.base = bBase_.as<int32_t>();
    v.big = bBig_.as<int32_t>();
    v.kbdone = bKbDone_.as<int32_t>();
    v.next = bNext_.as<int32_t>();
    v.hash = bHash_.as<int32_t>();
    v.ns = bNs_.as<int32_t>();
    v.phase = bPhase_.as<int32_t>();
    v.cont = bCont_.as<int32_t>();
    v.passes = bPasses_.as<int32_t>();
    v.total_passes = bTotPasses_.as<int32_t>();
    v.outer = bOuter_.as<int32_t>();
    v.err = bErr_.as<int32_t>();
    v.pairs = bPairs_.as<unsigned long long>();
    v.ctr = bCtr_.as<int32_t>();
    v.act_cloud = bActCloud_.as<int32_t>();
    v.act_pre = bActPre_.as<int32_t>();
    v.group_conv = bGroupConv_.as<int32_t>();
    v.ready = bReady_.as<int32_t>();
    v.dx = bDx_.as<float>();
    v.dcell = bDcell_.as<int32_t>();
    v.dalive = bDalive_.as<int32_t>();
    v.dc1 = bDc1_.as<int32_t>();
    v.dc2 = bDc2_.as<int32_t>();
    v.dbstart = bDbstart_.as<int32_t>();
    v.ditems = bDitems_.as<int32_t>();
    v.dnb_off = bDnbOff_.as<int32_t>();
    v.dnb = bDnb_.as<int32_t>();
    v.dbig = bDbig_.as<int32_t>();
    v.dcpre = bDcpre_.as<int32_t>();
    v.dec_smem_max = dec_smem_max_;
    v.dec_nb_pp = dec_nb_pp_;
    v.dec_hoff = bDecHoff_.as<int64_t>();
    v.dec_hbits = bDecHbits_.as<int32_t>();
    v.n_clouds = (int32_t)h_cl_.size();
    v.n_groups = (int32_t)h_gr_.size();
    v.n_chunks = n_chunks_;
    v.n_slots = n_slots_;
    v.n_kblk = n_kblk_;
    v.n_kblk_warp = n_kblk_warp_;
    v.chunk_pts = chunk_pts_;
    v.chunk_max = chunk_max_;
    v.hist_smem = hist_smem_;
    v.scat_smem = scat_smem_;
    v.max_passes = max_passes;
    v.max_outer = max_outer;
    v.max_iters = max_iters;
    v.Ps = bPs_.as<float>();
    v.sorder = bSorder_.as<int32_t>();
    v.srow = bSorder_.as<int32_t>() + total_points_;  // second half of the same buffer
    v.cull = cull_ ? 1 : 0;
    v.tile_order = bTileOrder_.as<int32_t>();
    v.n_heavy = n_heavy_;
    v.tile_cl_grid = tile_cl_grid_;
    v.tile_seg_min = tile_seg_min_;
    v.n_sms = sms_;
    v.flags = flags_;
    return v;
}

static int ceil_log2(int64_t x)
{
    int b = 0;
    while ((int64_t(1) << b) < x) ++b;
    return b;
}

int Engine::finish_setup_after_choose(cudaStream_t st)
{
    const size_t nc = h_cl_.size();
    h_ns_.resize(nc);
    if (DevArena* a = current_arena(); a && a->measuring()) {
        // size planning: the counts the caller will give
        for (size_t c = 0; c < nc; ++c) h_ns_[c] = c < given_ns.size() ? given_ns[c] : h_cl_[c].n_own;
    } else {
        RD_CK(cudaMemcpyAsync(h_ns_.data(), bNs_.p, 4 * nc, cudaMemcpyDeviceToHost, st));
        RD_CK(cudaStreamSynchronize(st));
    }
    int64_t hist = 0, key = 0, kblk = 0, kblk_warp = 0;
    int max_ns = 0;
    h_slot_cloud_.clear();
    for (size_t c = 0; c < nc; ++c) {
        CloudDesc& cd = h_cl_[c];
        cd.ns_cap = h_ns_[c];
        max_ns = std::max(max_ns, cd.ns_cap);
        cd.hist_off = hist;
        hist += (int64_t)cd.n_chunks * cd.ns_cap;
        cd.key_off = key;
        key += cd.ns_cap;
        (cd.n_chunks > SCAN_ROWS_WARP ? kblk : kblk_warp) += (cd.ns_cap + KBLK - 1) / KBLK;
        for (int k = 0; k < cd.ns_cap; ++k) h_slot_cloud_.push_back((int32_t)c);
    }
    n_slots_ = (int32_t)key;
    hist_ints_ = hist;
    n_kblk_ = (int32_t)kblk;
    n_kblk_warp_ = (int32_t)kblk_warp;
    // group decimation scratch
    h_dec_hoff_.resize(h_gr_.size());
    h_dec_hbits_.resize(h_gr_.size());
    int64_t sscr = 0, hoff = 0, max_tot = 0;
    for (size_t g = 0; g < h_gr_.size(); ++g) {
        GroupDesc& gd = h_gr_[g];
        int64_t tot = 0;
        for (int i = 0; i < gd.n_clouds; ++i) tot += h_cl_[gd.cloud_begin + i].ns_cap;
        gd.s_scratch = sscr;
        gd.s_cap = (int32_t)tot;
        sscr += tot;
        max_tot = std::max(max_tot, tot);
        const int hb = std::min(20, std::max(6, ceil_log2(std::max<int64_t>(tot, 1))));
        h_dec_hbits_[g] = hb;
        h_dec_hoff_[g] = hoff;
        hoff += (int64_t(1) << hb) + 1;
    }
    // shared-memory budgets (ints)
    hist_smem_ = std::min(max_ns, 24 * 1024);
    scat_smem_ = std::min(max_ns, 4 * 1024);
    RD_CK(upload(bCl_, h_cl_, st));
    RD_CK(upload(bGr_, h_gr_, st));
    RD_CK(upload(bSlotCloud_, h_slot_cloud_, st));
    RD_CK(upload(bDecHoff_, h_dec_hoff_, st));
    RD_CK(upload(bDecHbits_, h_dec_hbits_, st));
    RD_CK(bHist_.ensure(4 * (size_t)(hist + 1)));
    RD_CK(bCnt_.ensure(4 * (size_t)(key + 1)));
    RD_CK(bBase_.ensure(4 * (size_t)(key + 1)));
    RD_CK(bBig_.ensure(4 * (size_t)(key + 1)));
    RD_CK(bDx_.ensure(4 * (size_t)(sscr * dim_ + 1)));
    RD_CK(bDcell_.ensure(4 * (size_t)(sscr * dim_ + 1)));
    RD_CK(bDalive_.ensure(4 * (size_t)(sscr + 1)));
    RD_CK(bDc1_.ensure(4 * (size_t)(sscr + 1)));
    RD_CK(bDc2_.ensure(4 * (size_t)(sscr + 1)));
    RD_CK(bDitems_.ensure(4 * (size_t)(sscr + 1)));
    RD_CK(bDbstart_.ensure(4 * (size_t)(hoff + 1)));
    RD_CK(bDnbOff_.ensure(4 * (size_t)(sscr + h_gr_.size() + 1)));
    dec_nb_pp_ = (int)std::max<int64_t>(
        DEC_NB_MIN_PER_POINT,
        std::min<int64_t>(DEC_NB_MAX_PER_POINT, DEC_NB_BUDGET / std::max<int64_t>(sscr, 1)));
    RD_CK(bDnb_.ensure(4 * (size_t)((int64_t)dec_nb_pp_ * sscr + 1)));
    dec_smem_max_ = (int)std::min<int64_t>(max_tot, DEC_SMEM_MAX_POINTS);
    // persistent assignment grid: every resident CTA slot, at most one per chunk
    int dev = 0, sms = 0;
    RD_CK(cudaGetDevice(&dev));
    RD_CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    const int per_sm = std::max(1, max_assign_blocks_per_sm(dim_, tune, hist_smem_));
    assign_grid_ = std::max(1, std::min(n_chunks_, sms * per_sm));
    return 0;
}

int Engine::build_graph(cudaStream_t st)
{
    (void)st;
    const EngineView v = view();
    std::vector<unsigned char> key(sizeof(v) + sizeof(TuneParams) + 2 * sizeof(int));
    const int fz = fused_ ? 1 : 0;
    std::memcpy(key.data(), &v, sizeof(v));
    std::memcpy(key.data() + sizeof(v), &tune, sizeof(TuneParams));
    std::memcpy(key.data() + sizeof(v) + sizeof(TuneParams), &assign_grid_, sizeof(int));
    std::memcpy(key.data() + sizeof(v) + sizeof(TuneParams) + sizeof(int), &fz, sizeof(int));
    if (exec_ && key == graph_key_) return 0;
    if (exec_) { cudaGraphExecDestroy(exec_); exec_ = nullptr; }
    if (graph_) { cudaGraphDestroy(graph_); graph_ = nullptr; }
    if (!cap_stream_) RD_CK(cudaStreamCreateWithFlags(&cap_stream_, cudaStreamNonBlocking));
    RD_CK(cudaGraphCreate(&graph_, 0));
    cudaGraphConditionalHandle h;
    RD_CK(cudaGraphConditionalHandleCreate(&h, graph_, 1, cudaGraphCondAssignDefault));
    alignas(cudaGraphNodeParams) unsigned char cp_raw[sizeof(cudaGraphNodeParams)];
    std::memset(cp_raw, 0, sizeof(cp_raw));
    cudaGraphNodeParams& cp = *reinterpret_cast<cudaGraphNodeParams*>(cp_raw);
    cp.type = cudaGraphNodeTypeConditional;
    cp.conditional.handle = h;
    cp.conditional.type = cudaGraphCondTypeWhile;
    cp.conditional.size = 1;
    cudaGraphNode_t node;
    RD_CK(cudaGraphAddNode(&node, graph_, nullptr, 0, &cp));
    cudaGraph_t body = cp.conditional.phGraph_out[0];
    RD_CK(cudaStreamBeginCaptureToGraph(cap_stream_, body, nullptr, nullptr, 0,
                                        cudaStreamCaptureModeThreadLocal));
    LoopCond lc;
    lc.h = h;
    lc.use_handle = 1;
    cudaError_t e1 = fused_ ? launch_tile_pass(dim_, v, lc, cap_stream_)
                            : launch_pass(dim_, v, tune, assign_grid_, lc, cap_stream_);
    cudaGraph_t out = nullptr;
    cudaError_t e3 = cudaStreamEndCapture(cap_stream_, &out);
    if (e1 != cudaSuccess) return fail("capture pass", e1);
    if (e3 != cudaSuccess) return fail("end capture", e3);
    RD_CK(cudaGraphInstantiate(&exec_, graph_, 0));
    graph_key_ = key;
    return 0;
}

int Engine::run(cudaStream_t st, bool use_graph, int mode)
{
    if (h_cl_.empty()) return 0;
    stats_ = RunStats();
    flags_ = (mode == RUN_EVOLVE_ONLY) ? ENG_EVOLVE_ONLY : 0;
    RD_CK(upload(bCl_, h_cl_, st));
    RD_CK(upload(bGr_, h_gr_, st));
    RD_CK(upload(bChunkCloud_, h_chunk_cloud_, st));
    build_tile_order();
    RD_CK(upload(bTileOrder_, h_tile_order_, st));
    if (mode == RUN_EVOLVE_ONLY || mode == RUN_DECIMATE_ONLY) {
        // chosen sets supplied by the caller (given_ns, points already in S)
        if (given_ns.size() != h_cl_.size()) {
            last_error = "given chosen counts do not match the clouds";
            return 1;
        }
        for (size_t c = 0; c < h_cl_.size(); ++c)
            if (given_ns[c] < 0 || given_ns[c] > h_cl_[c].n_own) {
                last_error = "given chosen count exceeds the cloud's capacity";
                return 1;
            }
        EngineView v0 = view();
        RD_CK(launch_reset(v0, st));
        RD_CK(cudaMemcpyAsync(bNs_.p, given_ns.data(), 4 * given_ns.size(),
                              cudaMemcpyHostToDevice, st));
        if (int rc = finish_setup_after_choose(st)) return rc;
        const EngineView v1 = view();
        RD_CK(launch_set_given(v1, mode == RUN_DECIMATE_ONLY ? 1 : 0, st));
        if (mode == RUN_DECIMATE_ONLY) {
            RD_CK(launch_decimate(dim_, v1, st));
            return collect(st);
        }
    } else {
        // one large cloud: GPU-wide choose rounds; otherwise one CTA per cloud
        const bool rounds = h_cl_.size() == 1 && h_cl_[0].n_own >= (1 << 16);
        if (rounds) {
            RD_CK(bHash_.ensure(4 * (size_t)choose_hash_buckets()));
            RD_CK(bSurv_.ensure((size_t)h_cl_[0].n_own + 16));
            RD_CK(bSel_.ensure(4 * (size_t)(h_cl_[0].n_own + 2)));
            RD_CK(bSelTmp_.ensure(choose_select_scratch_bytes(h_cl_[0].n_own)));
        }
        EngineView v0 = view();
        RD_CK(launch_reset(v0, st));
        if (rounds)
            RD_CK(launch_choose_rounds(dim_, v0, 0, h_cl_[0].n_own, bSurv_.as<uint8_t>(),
                                       bSel_.as<int32_t>(), bSelTmp_.p, bSelTmp_.bytes, st));
        else
            RD_CK(launch_choose(dim_, v0, st));
        if (mode == RUN_CHOOSE_ONLY) {
            h_ns_.resize(h_cl_.size());
            RD_CK(cudaMemcpyAsync(h_ns_.data(), bNs_.p, 4 * h_ns_.size(), cudaMemcpyDeviceToHost,
                                  st));
            RD_CK(cudaStreamSynchronize(st));
            return 0;
        }
        if (int rc = finish_setup_after_choose(st)) return rc;
    }
    // Tiled runs (one group of many clouds, every chosen set small enough)
    // evolve each tile to convergence inside one kernel; everything else runs
    // lockstep passes over all evolving clouds.
    int max_ns = 0;
    for (const CloudDesc& cd : h_cl_) max_ns = std::max(max_ns, cd.ns_cap);
    fused_ = fuse_tiles && h_gr_.size() == 1 && h_cl_.size() > 1 && max_ns <= TILE_NS_MAX &&
             flags_ == 0;
    cull_ = cull_assign && assign_cull_enabled() && !fused_ && spatial_ok_ && total_points_ > 0;
    if (cull_) {
        const size_t scratch = spatial_prep_scratch_bytes(total_points_);
        RD_CK(bPs_.ensure(sizeof(float) * (size_t)(total_points_ * pad_dim(dim_) + 4)));
        RD_CK(bSorder_.ensure(sizeof(int32_t) * (size_t)(2 * total_points_ + 1)));
        RD_CK(bSpatialTmp_.ensure(scratch));
        const EngineView vs = view();
        RD_CK(launch_spatial_prep(dim_, vs, total_points_, bSpatialTmp_.p, scratch, bPs_.as<float>(),
                                  bSorder_.as<int32_t>(), st));
        // the culled assignment adds its counts into the histogram rows, which
        // k_scatter_cta zeroes again after every pass
        RD_CK(cudaMemsetAsync(bHist_.p, 0, 4 * (size_t)(hist_ints_ + 1), st));
    }
    tile_cl_grid_ = 0;
    if (fused_) RD_CK(prepare_tile_pass(dim_, view(), &tile_cl_grid_));
    const EngineView v = view();
    RD_CK(prepare_pass(dim_, v, tune));
    // work lists of the first iteration
    RD_CK(launch_loopcond(v, cudaGraphConditionalHandle(), 0, st, 0));
    if (use_graph) {
        if (int rc = build_graph(st)) return rc;
        RD_CK(cudaGraphLaunch(exec_, st));
    } else {
        cudaEvent_t a0 = nullptr, a1 = nullptr;
        if (profile_assign || profile_pass) {
            RD_CK(cudaEventCreate(&a0));
            RD_CK(cudaEventCreate(&a1));
        }
        stats_.assign_ms = 0;
        stats_.assign_launches = 0;
        for (;;) {
            // profile_pass: the events bracket the whole iteration instead of
            // the assignment kernel
            cudaEvent_t k0 = profile_pass ? nullptr : a0, k1 = profile_pass ? nullptr : a1;
            if (profile_pass) RD_CK(cudaEventRecord(a0, st));
            const LoopCond lc;  // no handle: the count is read below
            if (fused_) RD_CK(launch_tile_pass(dim_, v, lc, st, k0, k1));
            else RD_CK(launch_pass(dim_, v, tune, assign_grid_, lc, st, k0, k1));
            if (profile_pass) RD_CK(cudaEventRecord(a1, st));
            int32_t act = 0;
            RD_CK(cudaMemcpyAsync(&act, v.ctr + CTR_ACTIVE, 4, cudaMemcpyDeviceToHost, st));
            RD_CK(cudaStreamSynchronize(st));
            if (a0) {
                float ms = 0;
                RD_CK(cudaEventElapsedTime(&ms, a0, a1));
                stats_.assign_ms += ms;
                stats_.assign_launches += 1;
            }
            if (act == 0) break;
        }
        if (a0) cudaEventDestroy(a0);
        if (a1) cudaEventDestroy(a1);
    }
    return collect(st);
}

// Tiles (clouds) by decreasing evolve points; the heavy ones (evolved by a
// whole cluster in fused tiled runs) first.
void Engine::build_tile_order()
{
    const size_t nc = h_cl_.size();
    h_tile_order_.resize(nc);
    for (size_t c = 0; c < nc; ++c) h_tile_order_[c] = (int32_t)c;
    std::stable_sort(h_tile_order_.begin(), h_tile_order_.end(),
                     [&](int32_t a, int32_t b) { return h_cl_[a].n_all > h_cl_[b].n_all; });
    n_heavy_ = 0;
    const TileClusterParams tp = tile_cluster_params();
    tile_seg_min_ = std::max(1, tp.seg_min);
    if (tp.enabled && nc > 1)
        while (n_heavy_ < (int)nc && h_cl_[h_tile_order_[n_heavy_]].n_all >= tp.min_points)
            ++n_heavy_;
}

int Engine::plan_workspace(int mode)
{
    DevArena* a = current_arena();
    if (!a || !a->measuring()) {
        last_error = "workspace planning needs a measuring arena";
        return 1;
    }
    // the buffers run() takes, in its order, for a single-cloud device step
    RD_CK(upload(bCl_, h_cl_, nullptr));
    RD_CK(upload(bGr_, h_gr_, nullptr));
    RD_CK(upload(bChunkCloud_, h_chunk_cloud_, nullptr));
    build_tile_order();
    RD_CK(upload(bTileOrder_, h_tile_order_, nullptr));
    if (mode == RUN_EVOLVE_ONLY || mode == RUN_DECIMATE_ONLY) {
        if (int rc = finish_setup_after_choose(nullptr)) return rc;
        if (mode == RUN_EVOLVE_ONLY && cull_assign && assign_cull_enabled() && spatial_ok_ &&
            total_points_ > 0) {
            RD_CK(bPs_.ensure(sizeof(float) * (size_t)(total_points_ * pad_dim(dim_) + 4)));
            RD_CK(bSorder_.ensure(sizeof(int32_t) * (size_t)(2 * total_points_ + 1)));
            RD_CK(bSpatialTmp_.ensure(spatial_prep_scratch_bytes(total_points_)));
        }
        return 0;
    }
    if (mode == RUN_CHOOSE_ONLY) {
        if (h_cl_.size() == 1 && h_cl_[0].n_own >= (1 << 16)) {
            RD_CK(bHash_.ensure(4 * (size_t)choose_hash_buckets()));
            RD_CK(bSurv_.ensure((size_t)h_cl_[0].n_own + 16));
            RD_CK(bSel_.ensure(4 * (size_t)(h_cl_[0].n_own + 2)));
            RD_CK(bSelTmp_.ensure(choose_select_scratch_bytes(h_cl_[0].n_own)));
        }
        return 0;
    }
    last_error = "workspace planning covers the choose, evolve and decimate steps only";
    return 1;
}

int Engine::adjoint_setup(cudaStream_t st)
{
    if (h_cl_.size() != 1 || given_ns.size() != 1) {
        last_error = "adjoint: one cloud with a given chosen set";
        return 1;
    }
    if (given_ns[0] < 1 || given_ns[0] > h_cl_[0].n_own) {
        last_error = "adjoint: chosen count out of range";
        return 1;
    }
    stats_ = RunStats();
    flags_ = ENG_ALWAYS_MOVE;
    cull_ = false;
    RD_CK(upload(bCl_, h_cl_, st));
    RD_CK(upload(bGr_, h_gr_, st));
    EngineView v0 = view();
    RD_CK(launch_reset(v0, st));
    RD_CK(cudaMemcpyAsync(bNs_.p, given_ns.data(), 4, cudaMemcpyHostToDevice, st));
    if (int rc = finish_setup_after_choose(st)) return rc;
    const EngineView v = view();
    RD_CK(launch_set_given(v, 0, st));
    RD_CK(prepare_pass(dim_, v, tune));
    return 0;
}

int Engine::adjoint_step(cudaStream_t st)
{
    const EngineView v = view();
    RD_CK(launch_loopcond(v, cudaGraphConditionalHandle(), 0, st, 0));  // lists + ticket
    RD_CK(launch_evolve_step(dim_, v, tune, assign_grid_, st));
    return 0;
}

int Engine::collect(cudaStream_t st)
{
    const size_t nc = h_cl_.size();
    std::vector<int32_t> tp(nc);
    std::vector<unsigned long long> pr(nc);
    int32_t ctr[CTR_COUNT];
    h_err_.resize(nc);
    RD_CK(cudaMemcpyAsync(h_ns_.data(), bNs_.p, 4 * nc, cudaMemcpyDeviceToHost, st));
    RD_CK(cudaMemcpyAsync(h_err_.data(), bErr_.p, 4 * nc, cudaMemcpyDeviceToHost, st));
    RD_CK(cudaMemcpyAsync(tp.data(), bTotPasses_.p, 4 * nc, cudaMemcpyDeviceToHost, st));
    RD_CK(cudaMemcpyAsync(pr.data(), bPairs_.p, 8 * nc, cudaMemcpyDeviceToHost, st));
    RD_CK(cudaMemcpyAsync(ctr, bCtr_.p, sizeof(ctr), cudaMemcpyDeviceToHost, st));
    RD_CK(cudaStreamSynchronize(st));
    stats_.loop_iters = ctr[CTR_ITERS];
    stats_.err_bits = ctr[CTR_ERR];
    stats_.dec_passes = ctr[CTR_DEC_PASSES];
    stats_.dec_rounds = ctr[CTR_DEC_ROUNDS];
    for (size_t c = 0; c < nc; ++c) {
        stats_.total_passes += tp[c];
        stats_.max_passes = std::max<int64_t>(stats_.max_passes, tp[c]);
        stats_.pairs += (double)pr[c];
        stats_.point_passes += (double)h_cl_[c].n_all * (double)tp[c];
        stats_.err_bits |= h_err_[c];
    }
    if (stats_.err_bits & (ERRB_EVOLVE_CAP | ERRB_OUTER_CAP | ERRB_DEC_CAP)) {
        last_error = "iteration limit reached before convergence";
        return 4;  // RD_ERR_NOT_CONVERGED
    }
    if (stats_.err_bits & ERRB_CAPACITY) {
        last_error = "device capacity exceeded";
        return 3;
    }
    return 0;
}

}  // namespace rdb
