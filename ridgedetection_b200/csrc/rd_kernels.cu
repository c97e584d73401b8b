// rd_kernels.cu -- sm_100a kernels of the batch engine (see rd_engine.cuh).
//
// All arithmetic is FP32 on the CUDA cores.  The point/chosen contraction has
// K = DIM <= 3, far too thin for tcgen05 tiles, and the reference's rounding
// (sub, mul, add, each rounded) rules out the |p|^2 - 2 p.c + |c|^2 expansion a
// tensor-core formulation would need, so the hot loop is a register-blocked
// SIMT kernel instead: each thread holds ITEMS cloud points, the chosen set
// streams through shared memory, and every pair costs DIM sub + DIM mul +
// (DIM-1) add + compare + 2 selects, all explicitly rounded.
#include "rd_engine.cuh"
#include "rd_grid.cuh"
#include "rd_fold.cuh"
#include "rd_segfold.cuh"

#include <cuda_runtime.h>
#include <cub/cub.cuh>

#include <algorithm>
#include <atomic>
#include <cstring>

namespace rdb {

namespace {

// members from which a key is folded by a whole CTA of k_sum_shift (the
// warp-segmented exact fold of rd_segfold.cuh) instead of by one warp's add
// chain -- while the pass has at most two such keys per big-key CTA; with more
// (a batch of large clouds) every key is folded by a warp, which keeps all
// SMs busy.
constexpr int SUM_BIG_MIN = 16384;
constexpr int SUM_BIG_PER_CTA = 2;

// Programmatic dependent launch: the loop-body kernels are launched with
// programmatic stream serialisation, so a kernel's CTAs may become resident
// while the previous kernel drains. Each waits here, before its first access
// to memory, until the previous grid has completed and its writes are
// visible, then lets the next kernel launch. Launched without the attribute,
// both instructions return at once.
__device__ __forceinline__ void pdl_enter()
{
    asm volatile("griddepcontrol.wait;" ::: "memory");
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}

// Work lists over the clouds still evolving, rebuilt by k_loopcond after every
// iteration: act_cloud[a] is the a-th evolving cloud and act_pre[kind] the
// exclusive prefix of its work items (ACT_* in rd_engine.cuh), so kernels
// launched over fixed grids touch only active work.

struct ActiveList {
    const int32_t* pre;
    const int32_t* cloud;
    int nact;
    int total;
    __device__ ActiveList(const EngineView& v, int kind)
    {
        nact = v.ctr[CTR_NACT];
        pre = v.act_pre + (int64_t)kind * (v.n_clouds + 1);
        cloud = v.act_cloud;
        total = pre[nact];
    }
    // item t < total -> (cloud, item index inside that cloud)
    __device__ __forceinline__ void locate(int t, int& c, int& local) const
    {
        int lo = 0, hi = nact - 1;
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (pre[mid] <= t) lo = mid;
            else hi = mid - 1;
        }
        c = cloud[lo];
        local = t - pre[lo];
    }
};


// ---------------------------------------------------------------------------
// choose: rd/cpu/brute_force/choose.hpp:37-70, one CTA per cloud.
// Blocks of BLOCK points are visited in order.  Phase 1 (all threads) drops
// every point that has a chosen point within r1 among those chosen by earlier
// blocks, looked up through a hashed grid of cell edge > r1 (the grid only
// prunes; the test itself is the exact FP32 one).  Phase 2 (warp 0) walks the
// survivors in order and re-tests each against the grid, which by then also
// holds the points chosen earlier in the same block, so the outcome is the
// sequential greedy one.  Chosen coordinates and hash chains are mirrored in
// shared memory for the first SCAP chosen points.
// ---------------------------------------------------------------------------
template <int DIM>
struct ChooseSmem {
    static constexpr int HBITS = 13;
    static constexpr int HB = 1 << HBITS;
    static constexpr int SCAP = (DIM <= 2) ? 6144 : 4096;
};

template <int DIM, int BLOCK>
__global__ void __launch_bounds__(BLOCK) k_choose(EngineView v)
{
    using CS = ChooseSmem<DIM>;
    constexpr int NB = Pow3<DIM>::v;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    int32_t* s_heads = reinterpret_cast<int32_t*>(smem_raw);          // HB
    int32_t* s_next = s_heads + CS::HB;                                // SCAP
    float* s_S = reinterpret_cast<float*>(s_next + CS::SCAP);          // SCAP*DIM
    float* s_sp = s_S + CS::SCAP * DIM;                                // BLOCK*DIM
    int32_t* s_scell = reinterpret_cast<int32_t*>(s_sp + BLOCK * DIM); // BLOCK*DIM
    __shared__ int s_ns;
    __shared__ int s_wsum[BLOCK / 32];

    const int c = blockIdx.x;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const CloudDesc cd = v.cl[c];
    const int n = cd.n_own;
    const float rsq = sqr_rn(cd.r1);
    const double inv = 1.0 / ((double)cd.r1 * (1.0 + 1.0 / 1024.0));
    const uint32_t hmask = CS::HB - 1;
    float* gS = v.S + cd.s_off * DIM;
    int32_t* gnext = v.next + cd.s_off;
    const float* P = v.P + cd.p_off * DIM;

    for (int h = tid; h < CS::HB; h += BLOCK) s_heads[h] = -1;
    if (tid == 0) s_ns = 0;
    __syncthreads();

    auto coord = [&](int q, int d) -> float {
        return (q < CS::SCAP) ? s_S[q * DIM + d] : gS[(int64_t)q * DIM + d];
    };
    auto nxt = [&](int q) -> int { return (q < CS::SCAP) ? s_next[q] : gnext[q]; };
    // any chosen point within r1 of p, over the given neighbour cells
    auto query = [&](const float* p, const int* cc, int o) -> bool {
        int nc[DIM];
        neighbour_cell<DIM>(cc, o, nc);
        int q = s_heads[cell_hash<DIM>(nc) & hmask];
        while (q >= 0) {
            float s[DIM];
#pragma unroll
            for (int d = 0; d < DIM; ++d) s[d] = coord(q, d);
            if (sqdist_exact<DIM>(p, s) <= rsq) return true;
            q = nxt(q);
        }
        return false;
    };

    for (int base = 0; base < n; base += BLOCK) {
        const int i = base + tid;
        const bool valid = i < n;
        float p[DIM];
        int cc[DIM];
        bool surv = false;
        if (valid) {
#pragma unroll
            for (int d = 0; d < DIM; ++d) {
                p[d] = P[(int64_t)i * DIM + d];
                cc[d] = cell_of(p[d], inv);
            }
            bool hit = false;
            for (int t = 0; t < NB && !hit; ++t) hit = query(p, cc, (t + NB / 2) % NB);
            surv = !hit;
        }
        // compact survivors in visiting order
        const unsigned bal = __ballot_sync(FULL, surv);
        if (lane == 0) s_wsum[warp] = __popc(bal);
        __syncthreads();
        int wbase = 0, tot = 0;
        for (int w = 0; w < BLOCK / 32; ++w) {
            const int x = s_wsum[w];
            wbase += (w < warp) ? x : 0;
            tot += x;
        }
        if (surv) {
            const int pos = wbase + __popc(bal & lanemask_lt());
#pragma unroll
            for (int d = 0; d < DIM; ++d) {
                s_sp[pos * DIM + d] = p[d];
                s_scell[pos * DIM + d] = cc[d];
            }
        }
        __syncthreads();
        if (warp == 0) {
            int ns = s_ns;
            for (int sidx = 0; sidx < tot; ++sidx) {
                float ps[DIM];
                int cs[DIM];
#pragma unroll
                for (int d = 0; d < DIM; ++d) {
                    ps[d] = s_sp[sidx * DIM + d];
                    cs[d] = s_scell[sidx * DIM + d];
                }
                bool hit = false;
                for (int o = lane; o < NB; o += 32) hit = hit || query(ps, cs, o);
                hit = __any_sync(FULL, hit);
                if (!hit) {
                    if (lane == 0) {
                        const uint32_t b = cell_hash<DIM>(cs) & hmask;
                        const int head = s_heads[b];
#pragma unroll
                        for (int d = 0; d < DIM; ++d) gS[(int64_t)ns * DIM + d] = ps[d];
                        if (ns < CS::SCAP) {
#pragma unroll
                            for (int d = 0; d < DIM; ++d) s_S[ns * DIM + d] = ps[d];
                            s_next[ns] = head;
                        } else {
                            gnext[ns] = head;
                        }
                        s_heads[b] = ns;
                    }
                    ++ns;
                }
                __syncwarp();
            }
            if (lane == 0) s_ns = ns;
        }
        __syncthreads();
    }
    if (tid == 0) {
        v.ns[c] = s_ns;
        v.phase[c] = (s_ns > 0) ? PH_EVOLVE : PH_DONE;
    }
}

// ---------------------------------------------------------------------------
// choose for one large cloud, in rounds over growing ranges [a, b) of its
// points (same semantics as k_choose).  k_choose_filter, spread over the whole
// GPU, drops every point of the range that has a point chosen in earlier rounds
// within r1 (hash grid read from global memory); a stable compaction lists the
// survivors in order; k_choose_resolve, one CTA, walks that list and applies
// the sequential greedy rule with a shared-memory mirror of the grid, then
// writes the grid back for the next round's filter.
// ---------------------------------------------------------------------------
template <int DIM>
__global__ void __launch_bounds__(256) k_choose_filter(EngineView v, int c, int a, int b,
                                                       uint8_t* __restrict__ surv)
{
    using CS = ChooseSmem<DIM>;
    constexpr int NB = Pow3<DIM>::v;
    const CloudDesc cd = v.cl[c];
    const float rsq = sqr_rn(cd.r1);
    const double inv = 1.0 / ((double)cd.r1 * (1.0 + 1.0 / 1024.0));
    const uint32_t hmask = CS::HB - 1;
    const int32_t* heads = v.hash;
    const float* gS = v.S + cd.s_off * DIM;
    const int32_t* gnext = v.next + cd.s_off;
    const float* P = v.P + cd.p_off * DIM;
    for (int i = a + blockIdx.x * blockDim.x + threadIdx.x; i < b; i += gridDim.x * blockDim.x) {
        float p[DIM];
        int cc[DIM];
#pragma unroll
        for (int d = 0; d < DIM; ++d) {
            p[d] = P[(int64_t)i * DIM + d];
            cc[d] = cell_of(p[d], inv);
        }
        bool hit = false;
        for (int t = 0; t < NB && !hit; ++t) {
            int nc[DIM];
            neighbour_cell<DIM>(cc, (t + NB / 2) % NB, nc);
            for (int q = heads[cell_hash<DIM>(nc) & hmask]; q >= 0 && !hit; q = gnext[q]) {
                float s[DIM];
#pragma unroll
                for (int d = 0; d < DIM; ++d) s[d] = gS[(int64_t)q * DIM + d];
                hit = sqdist_exact<DIM>(p, s) <= rsq;
            }
        }
        surv[i - a] = hit ? 0 : 1;
    }
}

// sel: the survivors of [a, b) in order, *nsel of them (nullptr in the first
// round, where every point of the range is a candidate).  The candidates are
// taken in blocks of BLOCK as k_choose takes its points: all threads load
// their candidates, compute their cells and drop those within r1 of a point
// chosen so far (earlier rounds and earlier blocks of this one); warp 0 then
// walks the block's survivors in order, from shared memory.
template <int DIM, int BLOCK>
__global__ void __launch_bounds__(BLOCK) k_choose_resolve(EngineView v, int c, int a, int b,
                                                          const int32_t* __restrict__ sel,
                                                          const int32_t* __restrict__ nsel,
                                                          int first)
{
    using CS = ChooseSmem<DIM>;
    constexpr int NB = Pow3<DIM>::v;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    int32_t* s_heads = reinterpret_cast<int32_t*>(smem_raw);          // HB
    int32_t* s_next = s_heads + CS::HB;                                // SCAP
    float* s_S = reinterpret_cast<float*>(s_next + CS::SCAP);          // SCAP*DIM
    float* s_sp = s_S + CS::SCAP * DIM;                                // BLOCK*DIM
    int32_t* s_scell = reinterpret_cast<int32_t*>(s_sp + BLOCK * DIM); // BLOCK*DIM
    __shared__ int s_ns;
    __shared__ int s_wsum[BLOCK / 32];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const CloudDesc cd = v.cl[c];
    const float rsq = sqr_rn(cd.r1);
    const double inv = 1.0 / ((double)cd.r1 * (1.0 + 1.0 / 1024.0));
    const uint32_t hmask = CS::HB - 1;
    float* gS = v.S + cd.s_off * DIM;
    int32_t* gnext = v.next + cd.s_off;
    const float* P = v.P + cd.p_off * DIM;
    const int ns0 = first ? 0 : v.ns[c];
    for (int h = tid; h < CS::HB; h += BLOCK) s_heads[h] = first ? -1 : v.hash[h];
    for (int q = tid; q < min(ns0, CS::SCAP); q += BLOCK) {
        s_next[q] = gnext[q];
#pragma unroll
        for (int d = 0; d < DIM; ++d) s_S[q * DIM + d] = gS[(int64_t)q * DIM + d];
    }
    if (tid == 0) s_ns = ns0;
    __syncthreads();
    auto coord = [&](int q, int d) -> float {
        return (q < CS::SCAP) ? s_S[q * DIM + d] : gS[(int64_t)q * DIM + d];
    };
    auto nxt = [&](int q) -> int { return (q < CS::SCAP) ? s_next[q] : gnext[q]; };
    // any chosen point within r1 of p, over the given neighbour cells
    auto query = [&](const float* p, const int* cc, int o) -> bool {
        int nc[DIM];
        neighbour_cell<DIM>(cc, o, nc);
        int q = s_heads[cell_hash<DIM>(nc) & hmask];
        while (q >= 0) {
            float s[DIM];
#pragma unroll
            for (int d = 0; d < DIM; ++d) s[d] = coord(q, d);
            if (sqdist_exact<DIM>(p, s) <= rsq) return true;
            q = nxt(q);
        }
        return false;
    };
    const int cnt = sel ? *nsel : (b - a);
    for (int base = 0; base < cnt; base += BLOCK) {
        const int j = base + tid;
        float p[DIM];
        int cc[DIM];
        bool surv = false;
        if (j < cnt) {
            const int i = sel ? sel[j] : a + j;
#pragma unroll
            for (int d = 0; d < DIM; ++d) {
                p[d] = P[(int64_t)i * DIM + d];
                cc[d] = cell_of(p[d], inv);
            }
            bool hit = false;
            for (int t = 0; t < NB && !hit; ++t) hit = query(p, cc, (t + NB / 2) % NB);
            surv = !hit;
        }
        // compact the block's survivors in visiting order
        const unsigned bal = __ballot_sync(FULL, surv);
        if (lane == 0) s_wsum[warp] = __popc(bal);
        __syncthreads();
        int wbase = 0, tot = 0;
        for (int w = 0; w < BLOCK / 32; ++w) {
            const int x = s_wsum[w];
            wbase += (w < warp) ? x : 0;
            tot += x;
        }
        if (surv) {
            const int pos = wbase + __popc(bal & lanemask_lt());
#pragma unroll
            for (int d = 0; d < DIM; ++d) {
                s_sp[pos * DIM + d] = p[d];
                s_scell[pos * DIM + d] = cc[d];
            }
        }
        __syncthreads();
        if (warp == 0) {
            int ns = s_ns;
            for (int sidx = 0; sidx < tot; ++sidx) {
                float ps[DIM];
                int cs[DIM];
#pragma unroll
                for (int d = 0; d < DIM; ++d) {
                    ps[d] = s_sp[sidx * DIM + d];
                    cs[d] = s_scell[sidx * DIM + d];
                }
                bool hit = false;
                for (int o = lane; o < NB; o += 32) hit = hit || query(ps, cs, o);
                hit = __any_sync(FULL, hit);
                if (!hit) {
                    if (lane == 0) {
                        const uint32_t hb = cell_hash<DIM>(cs) & hmask;
                        const int head = s_heads[hb];
#pragma unroll
                        for (int d = 0; d < DIM; ++d) gS[(int64_t)ns * DIM + d] = ps[d];
                        gnext[ns] = head;
                        if (ns < CS::SCAP) {
#pragma unroll
                            for (int d = 0; d < DIM; ++d) s_S[ns * DIM + d] = ps[d];
                            s_next[ns] = head;
                        }
                        s_heads[hb] = ns;
                    }
                    ++ns;
                }
                __syncwarp();
            }
            if (lane == 0) s_ns = ns;
        }
        __syncthreads();
    }
    for (int h = tid; h < CS::HB; h += BLOCK) v.hash[h] = s_heads[h];
    if (tid == 0) {
        v.ns[c] = s_ns;
        v.phase[c] = (s_ns > 0) ? PH_EVOLVE : PH_DONE;
    }
}

// ---------------------------------------------------------------------------
// assign: rd/cpu/brute_force/evolve.hpp:43-66 over one chunk of CHUNK cloud
// points per work item; writes the key of every point and the chunk's key
// histogram row.  This is the hot kernel.
// ---------------------------------------------------------------------------
template <int DIM>
__device__ __forceinline__ void load_chosen(const float* sS, int kk, float* s)
{
    constexpr int DP = PadDim<DIM>::v;
    if constexpr (DP == 4) {
        const float4 t = reinterpret_cast<const float4*>(sS)[kk];
        s[0] = t.x; s[1] = t.y; s[2] = t.z;
        if constexpr (DIM == 4) s[3] = t.w;
    } else if constexpr (DP == 2) {
        const float2 t = reinterpret_cast<const float2*>(sS)[kk];
        s[0] = t.x; s[1] = t.y;
    } else {
#pragma unroll
        for (int d = 0; d < DIM; ++d) s[d] = sS[kk * DP + d];
    }
}

constexpr int ASSIGN_TS = 1024;  // chosen points per shared-memory tile

template <int DIM, int BLOCK, int ITEMS>
__global__ void __launch_bounds__(BLOCK) k_assign(EngineView v)
{
    pdl_enter();
    constexpr int DP = PadDim<DIM>::v;
    constexpr int TS = ASSIGN_TS;
    __shared__ __align__(16) float sS[TS * DP];
    __shared__ int s_item;
    extern __shared__ int s_hist[];
    const int tid = threadIdx.x;

    const ActiveList al(v, ACT_CHUNK);
    for (;;) {
        if (tid == 0) s_item = atomicAdd(&v.ctr[CTR_WORK], 1);
        __syncthreads();
        const int item = s_item;
        __syncthreads();
        if (item >= al.total) break;
        int c, lc;
        al.locate(item, c, lc);
        const CloudDesc cd = v.cl[c];
        // chunks split the cloud evenly (at most BLOCK*ITEMS points each)
        const int start = (int)(((int64_t)lc * cd.n_all) / cd.n_chunks);
        const int n = (int)(((int64_t)(lc + 1) * cd.n_all) / cd.n_chunks);  // chunk end
        const int ns = v.ns[c];
        const float* P = v.P + cd.p_off * DIM;
        const float* gS = v.S + cd.s_off * DIM;

        // Two-level argmin.  The inner loop keeps only the running minimum
        // (one min per pair instead of compare + two selects) and records the
        // block of KB chosen points in which it last decreased; the exact
        // index is then the first point of that block at exactly the minimum.
        // Strict decrease per block and first match inside the block give the
        // reference's rule: lowest index among equal minima.
        constexpr int KB = 8;
        constexpr float FAR = 1e30f;  // padding: (FAR - p)^2 overflows to +inf
        static_assert(ITEMS % 2 == 0, "points are processed in pairs");
        float p[ITEMS][DIM];
        float2 np2[ITEMS / 2][DIM];  // negated coordinates of point pairs (2jj, 2jj+1)
        float best[ITEMS];
        int blk[ITEMS];
#pragma unroll
        for (int j = 0; j < ITEMS; ++j) {
            const int i = start + j * BLOCK + tid;
#pragma unroll
            for (int d = 0; d < DIM; ++d) p[j][d] = (i < n) ? P[(int64_t)i * DIM + d] : 0.0f;
            best[j] = FLT_MAX;
            blk[j] = -1;
        }
#pragma unroll
        for (int jj = 0; jj < ITEMS / 2; ++jj)
#pragma unroll
            for (int d = 0; d < DIM; ++d) np2[jj][d] = make_float2(-p[2 * jj][d], -p[2 * jj + 1][d]);
        for (int t0 = 0; t0 < ns; t0 += TS) {
            const int tl = min(TS, ns - t0);
            const int tlp = (tl + KB - 1) / KB * KB;
            __syncthreads();
            for (int e = tid; e < tlp; e += BLOCK) {
#pragma unroll
                for (int d = 0; d < DIM; ++d)
                    sS[e * DP + d] = (e < tl) ? gS[(int64_t)(t0 + e) * DIM + d] : FAR;
            }
            __syncthreads();
            for (int kb = 0; kb < tlp; kb += KB) {
                float old[ITEMS];
#pragma unroll
                for (int j = 0; j < ITEMS; ++j) old[j] = best[j];
#pragma unroll
                for (int u = 0; u < KB; ++u) {
                    float s[DIM];
                    load_chosen<DIM>(sS, kb + u, s);
#pragma unroll
                    for (int jj = 0; jj < ITEMS / 2; ++jj) {
                        const float2 q = sqdist2_exact<DIM>(s, np2[jj]);
                        best[2 * jj] = fminf(best[2 * jj], q.x);
                        best[2 * jj + 1] = fminf(best[2 * jj + 1], q.y);
                    }
                }
#pragma unroll
                for (int j = 0; j < ITEMS; ++j) blk[j] = (best[j] < old[j]) ? (t0 + kb) : blk[j];
            }
        }
        const float rsq = sqr_rn(cd.r1);
        int key[ITEMS];
#pragma unroll
        for (int j = 0; j < ITEMS; ++j) {
            const int i = start + j * BLOCK + tid;
            int idx = -1;
            if (i < n && best[j] <= rsq && blk[j] >= 0) {
                for (int u = 0; u < KB; ++u) {
                    const int k = blk[j] + u;
                    if (k >= ns) break;
                    float s[DIM];
#pragma unroll
                    for (int d = 0; d < DIM; ++d) s[d] = gS[(int64_t)k * DIM + d];
                    if (sqdist_exact<DIM>(s, p[j]) == best[j]) { idx = k; break; }
                }
            }
            key[j] = idx;
            if (i < n) v.keys[cd.p_off + i] = key[j];
        }
        // chunk histogram row (row length ns_cap, first ns entries used)
        int32_t* row = v.hist + cd.hist_off + (int64_t)lc * cd.ns_cap;
        if (ns <= v.hist_smem) {
            for (int k = tid; k < ns; k += BLOCK) s_hist[k] = 0;
            __syncthreads();
#pragma unroll
            for (int j = 0; j < ITEMS; ++j)
                if (key[j] >= 0) atomicAdd(&s_hist[key[j]], 1);
            __syncthreads();
            for (int k = tid; k < ns; k += BLOCK) row[k] = s_hist[k];
        } else {
            for (int k = tid; k < ns; k += BLOCK) row[k] = 0;
            __syncthreads();
#pragma unroll
            for (int j = 0; j < ITEMS; ++j)
                if (key[j] >= 0) atomicAdd(&row[key[j]], 1);
        }
    }
}

// ---------------------------------------------------------------------------
// Culled assignment: the same keys as k_assign, over the spatial order (Ps,
// built once per run by launch_spatial_prep, DIM padded to PadDim) instead of
// the slot order.  A work item is a block of AC_BLOCK x AC_ITEMS consecutive
// points of that order; each warp takes 32 x AC_ITEMS of them and their
// bounding box.  A chosen point s takes part in a box's argmin only when the
// squared gap between s and the box, g2, is at most thr = r1^2 (1 + 2^-10)
// (rounded up).  Exactness: the computed g2 exceeds the exact squared gap G by
// at most a relative 2^-20 (a few roundings of non-negative terms), and every
// computed distance from s to a point of the box is at least G (1 - 2^-20);
// so g2 > thr makes every such distance > r1^2.  A skipped chosen point can
// then neither be the nearest one within r1 nor tie with it, and the minimum
// over the remaining points, visited in index order with strict '<', is the
// reference's (rd/cpu/brute_force/evolve.hpp:54-66).  The bound needs r1^2 in
// the normal range; any other r1 disables the skip.  NaN gaps never skip.
//
// The test runs at two levels.  The CTA's box (the union of its warps' boxes)
// is tested against every chosen point of the cloud, each thread taking a few
// of them; the survivors are compacted in index order into a shared list.
// The argument above holds for any box that contains the points, so a point
// dropped there is dropped for every warp.  Each warp then tests the short
// list against its own box and evaluates the distances of the kept chosen
// points, still in index order.  The chosen points stay staged in shared
// memory across the CTA's work items while they belong to one cloud of at
// most AC_TS chosen points.
//
// Keys are written back to the points' slots, and each assigned point adds
// one to its key's entry in the histogram row of its slot-order chunk (the
// rows k_assign writes itself; k_scatter_cta zeroes them again after use).
// ---------------------------------------------------------------------------
constexpr int AC_BLOCK = 256;             // threads of k_assign_cull
constexpr int AC_WARPS = AC_BLOCK / 32;
constexpr int AC_TS = 1024;               // chosen points per shared-memory batch
// points per lane (AC_ITEMS, a tuning parameter): a warp's box holds 32 x
// AC_ITEMS consecutive points of the spatial order

// squared gap between s and the box [lo, hi] (0 inside; NaN-free for NaN s)
template <int DIM>
__device__ __forceinline__ float box_gap2(const float* s, const float* lo, const float* hi)
{
    float g2 = 0.0f;
#pragma unroll
    for (int d = 0; d < DIM; ++d) {
        const float gap = fmaxf(fmaxf(__fsub_rn(lo[d], s[d]), __fsub_rn(s[d], hi[d])), 0.0f);
        g2 = __fadd_rn(g2, __fmul_rn(gap, gap));
    }
    return g2;
}

template <int DIM, int AC_ITEMS>
__global__ void __launch_bounds__(AC_BLOCK) k_assign_cull(EngineView v)
{
    pdl_enter();
    static_assert(AC_ITEMS % 2 == 0, "points are evaluated in pairs");
    constexpr int DP = PadDim<DIM>::v;
    constexpr int WPTS = 32 * AC_ITEMS;
    constexpr int SUBPTS = AC_BLOCK * AC_ITEMS;
    __shared__ __align__(16) float sS[AC_TS * DP];  // staged chosen batch
    __shared__ int sK[2][AC_TS];                     // CTA survivors: batch positions
    __shared__ float s_box[2][AC_WARPS][2 * DIM];    // warp boxes
    __shared__ float s_cbox[2][2 * DIM];             // the CTA's box
    __shared__ int s_wcnt[2][AC_WARPS];              // survivors per warp range
    __shared__ int s_staged;                         // cloud whose whole chosen set is in sS
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;

    const ActiveList al(v, ACT_CHUNK);
    // Each cloud is cut into blocks of SUBPTS consecutive positions of its
    // spatial order, `subs` blocks per assignment chunk (a power of two: both
    // sizes are); blocks past the cloud's end are empty.  The block bounds
    // need no division.
    const int subs = (v.chunk_pts + SUBPTS - 1) / SUBPTS;
    const int subs_log = 31 - __clz(subs);
    const int total = al.total * subs;

    // A work item's cloud, point range and this lane's points with their
    // slots and histogram rows; the next item's are loaded while the current
    // one is evaluated.
    struct Item {
        int c, b0, b1;
        float p[AC_ITEMS][DIM];
        int slot[AC_ITEMS], row[AC_ITEMS];
    };
    auto load_item = [&](const int item, Item& t) {
        t.c = -1;
        t.b0 = t.b1 = 0;
#pragma unroll
        for (int j = 0; j < AC_ITEMS; ++j) {
            t.slot[j] = -1;
            t.row[j] = 0;
#pragma unroll
            for (int d = 0; d < DIM; ++d) t.p[j][d] = 0.0f;
        }
        if (item >= total) return;
        int lc;
        al.locate(item >> subs_log, t.c, lc);
        const int n_all = v.cl[t.c].n_all;
        const int64_t p_off = v.cl[t.c].p_off;
        t.b0 = min(n_all, ((lc << subs_log) + (item & (subs - 1))) * SUBPTS);
        t.b1 = min(n_all, t.b0 + SUBPTS);
        const float* Ps = v.Ps + p_off * DP;
#pragma unroll
        for (int j = 0; j < AC_ITEMS; ++j) {
            const int i = t.b0 + warp * WPTS + j * 32 + lane;
            if (i < t.b1) {
                load_chosen<DIM>(Ps, i, t.p[j]);
                t.slot[j] = v.sorder[p_off + i];
                t.row[j] = v.srow[p_off + i];
            }
        }
    };

    if (tid == 0) s_staged = -1;
    // Items are dealt to the CTAs round robin (they are of equal size), so
    // every CTA knows its next item at once: its points are loaded while the
    // current one is evaluated.  Shared arrays indexed by `buf` alternate
    // between items, so a warp still reading the previous item's list never
    // races the next item's writes; sS is rewritten only after the barrier
    // that every warp reaches once it is done with the previous item.
    Item cur;
    load_item(blockIdx.x, cur);
    int it = 0;
    for (int item = blockIdx.x; item < total; item += gridDim.x, ++it) {
        const int buf = it & 1;
        Item nxt;
        load_item(item + gridDim.x, nxt);
        const int c = cur.c;
        const CloudDesc cd = v.cl[c];
        const int ns = v.ns[c];
        const float* gS = v.S + cd.s_off * DIM;
        const float rsq = sqr_rn(cd.r1);
        const bool may_skip = rsq >= 1.0e-30f && rsq <= 1.0e30f;
        const float thr = __fmul_ru(rsq, 1.0009765625f);

        // this warp's box (empty when the item has no points here)
        float blo[DIM], bhi[DIM];
#pragma unroll
        for (int d = 0; d < DIM; ++d) {
            blo[d] = INFINITY;
            bhi[d] = -INFINITY;
        }
#pragma unroll
        for (int j = 0; j < AC_ITEMS; ++j)
            if (cur.slot[j] >= 0)
#pragma unroll
                for (int d = 0; d < DIM; ++d) {
                    blo[d] = fminf(blo[d], cur.p[j][d]);
                    bhi[d] = fmaxf(bhi[d], cur.p[j][d]);
                }
#pragma unroll
        for (int d = 0; d < DIM; ++d) {
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
                blo[d] = fminf(blo[d], __shfl_xor_sync(FULL, blo[d], o));
                bhi[d] = fmaxf(bhi[d], __shfl_xor_sync(FULL, bhi[d], o));
            }
        }
        if (lane == 0) {
#pragma unroll
            for (int d = 0; d < DIM; ++d) {
                s_box[buf][warp][d] = blo[d];
                s_box[buf][warp][DIM + d] = bhi[d];
            }
        }
        float2 np2[AC_ITEMS / 2][DIM];
        float best[AC_ITEMS];
        int bi[AC_ITEMS];
#pragma unroll
        for (int jj = 0; jj < AC_ITEMS / 2; ++jj)
#pragma unroll
            for (int d = 0; d < DIM; ++d)
                np2[jj][d] = make_float2(-cur.p[2 * jj][d], -cur.p[2 * jj + 1][d]);
#pragma unroll
        for (int j = 0; j < AC_ITEMS; ++j) {
            best[j] = FLT_MAX;
            bi[j] = -1;
        }
        __syncthreads();  // warp boxes visible; the previous item is done
        if (warp == 0 && lane < 2 * DIM) {
            const bool hi = lane >= DIM;
            float x = s_box[buf][0][lane];
            for (int w = 1; w < AC_WARPS; ++w)
                x = hi ? fmaxf(x, s_box[buf][w][lane]) : fminf(x, s_box[buf][w][lane]);
            s_cbox[buf][lane] = x;
        }
        const bool cached = s_staged == c && ns <= AC_TS;
        for (int t0 = 0; t0 < ns; t0 += AC_TS) {
            const int tl = min(AC_TS, ns - t0);
            if (!(t0 == 0 && cached)) {
                if (t0 > 0) __syncthreads();  // the previous batch is no longer read
                for (int e = tid; e < tl; e += AC_BLOCK) {
                    float s[DIM];
#pragma unroll
                    for (int d = 0; d < DIM; ++d) s[d] = gS[(int64_t)(t0 + e) * DIM + d];
#pragma unroll
                    for (int d = 0; d < DIM; ++d) sS[e * DP + d] = s[d];
                }
            }
            __syncthreads();  // batch staged, CTA box known
            if (t0 == 0 && !cached && tid == 0) s_staged = (ns <= AC_TS) ? c : -1;
            float clo[DIM], chi[DIM];
#pragma unroll
            for (int d = 0; d < DIM; ++d) {
                clo[d] = s_cbox[buf][d];
                chi[d] = s_cbox[buf][DIM + d];
            }
            // CTA-level test: warp w takes batch positions [w*cw, (w+1)*cw)
            const int cw = ((tl + AC_BLOCK - 1) / AC_BLOCK) * 32;
            unsigned keepbits = 0;
            int wc = 0;
            for (int r = 0; r * 32 < cw; ++r) {
                const int e = warp * cw + r * 32 + lane;
                bool keep = false;
                if (e < tl) {
                    float s[DIM];
                    load_chosen<DIM>(sS, e, s);
                    keep = !(may_skip && box_gap2<DIM>(s, clo, chi) > thr);
                }
                keepbits |= keep ? (1u << r) : 0u;
                wc += __popc(__ballot_sync(FULL, keep));
            }
            if (lane == 0) s_wcnt[buf][warp] = wc;
            __syncthreads();
            int pos = 0, nk = 0;
#pragma unroll
            for (int w = 0; w < AC_WARPS; ++w) {
                const int x = s_wcnt[buf][w];
                pos += (w < warp) ? x : 0;
                nk += x;
            }
            for (int r = 0; r * 32 < cw; ++r) {
                const bool keep = (keepbits >> r) & 1u;
                const unsigned bal = __ballot_sync(FULL, keep);
                if (keep) sK[buf][pos + __popc(bal & ((1u << lane) - 1u))] = warp * cw + r * 32 + lane;
                pos += __popc(bal);
            }
            __syncthreads();
            // warp level: the survivors against this warp's box, then distances
            for (int q0 = 0; q0 < nk; q0 += 32) {
                const int q = q0 + lane;
                int e = 0;
                bool keep = false;
                if (q < nk) {
                    e = sK[buf][q];
                    float s[DIM];
                    load_chosen<DIM>(sS, e, s);
                    keep = !(may_skip && box_gap2<DIM>(s, blo, bhi) > thr);
                }
                unsigned bal = __ballot_sync(FULL, keep);
                // kept chosen points in index order, warp-uniform, two per
                // step: both distances are in flight together, and the
                // minimum is updated with the first one before the second
                while (bal) {
                    const int b1 = __ffs(bal) - 1;
                    bal &= bal - 1;
                    const bool two = bal != 0u;
                    const int b2 = two ? __ffs(bal) - 1 : b1;
                    bal &= bal - 1;
                    const int e1 = __shfl_sync(FULL, e, b1), e2 = __shfl_sync(FULL, e, b2);
                    float s1[DIM], s2[DIM];
                    load_chosen<DIM>(sS, e1, s1);
                    load_chosen<DIM>(sS, e2, s2);
                    const int k1 = t0 + e1, k2 = t0 + e2;
#pragma unroll
                    for (int jj = 0; jj < AC_ITEMS / 2; ++jj) {
                        const float2 d1 = sqdist2_exact<DIM>(s1, np2[jj]);
                        const float2 d2 = sqdist2_exact<DIM>(s2, np2[jj]);
                        if (d1.x < best[2 * jj]) { best[2 * jj] = d1.x; bi[2 * jj] = k1; }
                        if (d1.y < best[2 * jj + 1]) { best[2 * jj + 1] = d1.y; bi[2 * jj + 1] = k1; }
                        if (two && d2.x < best[2 * jj]) { best[2 * jj] = d2.x; bi[2 * jj] = k2; }
                        if (two && d2.y < best[2 * jj + 1]) { best[2 * jj + 1] = d2.y; bi[2 * jj + 1] = k2; }
                    }
                }
            }
        }
        int32_t* hist = v.hist + cd.hist_off;
#pragma unroll
        for (int j = 0; j < AC_ITEMS; ++j) {
            if (cur.slot[j] >= 0) {
                const int key = (best[j] <= rsq) ? bi[j] : -1;
                v.keys[cur.slot[j]] = key;
                if (key >= 0) atomicAdd(&hist[(int64_t)cur.row[j] * cd.ns_cap + key], 1);
            }
        }
        cur = nxt;
    }
}

// ---------------------------------------------------------------------------
// Chunk scan: for every chosen point k of a cloud, the exclusive prefix over
// the cloud's chunks of the chunk x key histogram (in place: afterwards row lc
// holds, for each key, the members in earlier chunks) and the member count
// cnt[k].  Work item = block of KBLK keys, one key per lane.
//   k_chunkscan_cta   clouds with more than SCAN_ROWS_WARP chunk rows: one CTA
//                     per item; the CS_W warps take contiguous row ranges, sum
//                     them, exchange the warp totals, and rescan their rows
//                     writing the prefixes;
//   k_chunkscan_warp  the other clouds: one warp per item, a single pass.
// The key bases follow in the same kernel: the CTA (warp) that finishes the
// last key block of a cloud -- a per-cloud counter of finished blocks says
// which -- forms the exclusive prefix of the cloud's member counts (each
// key's first grouped slot) and lists the keys of SUM_BIG_MIN or more members
// for the CTA-wide folds of k_sum_shift.
// ---------------------------------------------------------------------------
constexpr int CS_W = 16;   // warps of the CTA-wide scan
constexpr int CSW_W = 8;   // items (warps) per CTA of the warp-wide scan
constexpr int CS_LOADS = 16;  // histogram loads in flight per lane
constexpr int CS_REG = 32;    // rows per warp kept in registers between the two passes

// key bases of cloud c by the whole CTA (any multiple of 32 threads)
__device__ void key_bases_cta(const EngineView& v, const int c, int* s_w, int& s_carry)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    const CloudDesc cd = v.cl[c];
    const int ns = v.ns[c];
    const int32_t* cnt = v.cnt + cd.key_off;
    int32_t* base = v.base + cd.key_off;
    __syncthreads();  // earlier readers of s_w / s_carry are done
    if (threadIdx.x == 0) s_carry = 0;
    for (int k0 = 0; k0 < ns; k0 += blockDim.x) {
        __syncthreads();
        const int k = k0 + threadIdx.x;
        const int x = (k < ns) ? cnt[k] : 0;
        int incl = x;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(FULL, incl, o);
            if (lane >= o) incl += y;
        }
        if (lane == 31) s_w[warp] = incl;
        __syncthreads();
        int wpre = 0, tot = 0;
        for (int w = 0; w < nw; ++w) {
            wpre += (w < warp) ? s_w[w] : 0;
            tot += s_w[w];
        }
        const int carry = s_carry;
        if (k < ns) base[k] = carry + wpre + incl - x;
        if (x >= SUM_BIG_MIN) v.big[atomicAdd(&v.ctr[CTR_NBIG], 1)] = (int)(cd.key_off + k);
        __syncthreads();
        if (threadIdx.x == 0) s_carry = carry + tot;
    }
}

// the same by one warp
__device__ void key_bases_warp(const EngineView& v, const int c, const int lane)
{
    const CloudDesc cd = v.cl[c];
    const int ns = v.ns[c];
    const int32_t* cnt = v.cnt + cd.key_off;
    int32_t* base = v.base + cd.key_off;
    int carry = 0;
    for (int k0 = 0; k0 < ns; k0 += 32) {
        const int k = k0 + lane;
        const int x = (k < ns) ? cnt[k] : 0;
        int incl = x;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(FULL, incl, o);
            if (lane >= o) incl += y;
        }
        if (k < ns) base[k] = carry + incl - x;
        if (x >= SUM_BIG_MIN) v.big[atomicAdd(&v.ctr[CTR_NBIG], 1)] = (int)(cd.key_off + k);
        carry += __shfl_sync(FULL, incl, 31);
    }
}

__global__ void __launch_bounds__(CS_W * 32) k_chunkscan_cta(EngineView v)
{
    pdl_enter();
    __shared__ int s_part[CS_W][32];
    __shared__ int s_w[CS_W];
    __shared__ int s_carry, s_last;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const ActiveList al(v, ACT_KBLK);
    for (int item = blockIdx.x; item < al.total; item += gridDim.x) {
        int c, kb;
        al.locate(item, c, kb);
        const CloudDesc cd = v.cl[c];
        const int ns = v.ns[c];
        const int k = kb * KBLK + lane;
        const bool ok = k < ns;
        const int rows = cd.n_chunks;
        const int rw0 = (warp * rows) / CS_W, rw1 = ((warp + 1) * rows) / CS_W;
        int32_t* h = v.hist + cd.hist_off + k;
        // the first CS_REG rows of the warp's range stay in registers for the
        // rescan; longer ranges reload the rest
        int xr[CS_REG];
        int sum = 0;
#pragma unroll
        for (int u = 0; u < CS_REG; ++u)
            xr[u] = (ok && rw0 + u < rw1) ? h[(int64_t)(rw0 + u) * cd.ns_cap] : 0;
#pragma unroll
        for (int u = 0; u < CS_REG; ++u) sum += xr[u];
        for (int r0 = rw0 + CS_REG; r0 < rw1; r0 += CS_LOADS) {
            int x[CS_LOADS];
#pragma unroll
            for (int u = 0; u < CS_LOADS; ++u)
                x[u] = (ok && r0 + u < rw1) ? h[(int64_t)(r0 + u) * cd.ns_cap] : 0;
#pragma unroll
            for (int u = 0; u < CS_LOADS; ++u) sum += x[u];
        }
        s_part[warp][lane] = sum;
        __syncthreads();
        int run = 0, tot = 0;
#pragma unroll
        for (int w = 0; w < CS_W; ++w) {
            const int y = s_part[w][lane];
            run += (w < warp) ? y : 0;
            tot += y;
        }
#pragma unroll
        for (int u = 0; u < CS_REG; ++u) {
            if (ok && rw0 + u < rw1) h[(int64_t)(rw0 + u) * cd.ns_cap] = run;
            run += xr[u];
        }
        for (int r0 = rw0 + CS_REG; r0 < rw1; r0 += CS_LOADS) {
            int x[CS_LOADS];
#pragma unroll
            for (int u = 0; u < CS_LOADS; ++u)
                x[u] = (ok && r0 + u < rw1) ? h[(int64_t)(r0 + u) * cd.ns_cap] : 0;
#pragma unroll
            for (int u = 0; u < CS_LOADS; ++u) {
                if (ok && r0 + u < rw1) h[(int64_t)(r0 + u) * cd.ns_cap] = run;
                run += x[u];
            }
        }
        if (warp == 0 && ok) v.cnt[cd.key_off + k] = tot;
        // the last key block of the cloud: its key bases
        __threadfence();
        __syncthreads();  // also: s_part is reused by the next item
        if (threadIdx.x == 0)
            s_last = atomicAdd(&v.kbdone[c], 1) == (ns + KBLK - 1) / KBLK - 1;
        __syncthreads();
        if (s_last) {
            __threadfence();
            key_bases_cta(v, c, s_w, s_carry);
            if (threadIdx.x == 0) v.kbdone[c] = 0;
        }
    }
}

__global__ void __launch_bounds__(CSW_W * 32) k_chunkscan_warp(EngineView v)
{
    pdl_enter();
    const int lane = threadIdx.x & 31;
    const ActiveList al(v, ACT_KBLK_WARP);
    const int stride = gridDim.x * CSW_W;
    for (int item = blockIdx.x * CSW_W + (threadIdx.x >> 5); item < al.total; item += stride) {
        int c, kb;
        al.locate(item, c, kb);
        const CloudDesc cd = v.cl[c];
        const int ns = v.ns[c];
        const int k = kb * KBLK + lane;
        const bool ok = k < ns;
        const int rows = cd.n_chunks;
        int32_t* h = v.hist + cd.hist_off + k;
        int run = 0;
        for (int r0 = 0; r0 < rows; r0 += CS_LOADS) {
            int x[CS_LOADS];
#pragma unroll
            for (int u = 0; u < CS_LOADS; ++u)
                x[u] = (ok && r0 + u < rows) ? h[(int64_t)(r0 + u) * cd.ns_cap] : 0;
#pragma unroll
            for (int u = 0; u < CS_LOADS; ++u) {
                if (ok && r0 + u < rows) h[(int64_t)(r0 + u) * cd.ns_cap] = run;
                run += x[u];
            }
        }
        if (ok) v.cnt[cd.key_off + k] = run;
        // the last key block of the cloud: its key bases
        __threadfence();
        __syncwarp();
        int last = 0;
        if (lane == 0) last = atomicAdd(&v.kbdone[c], 1) == (ns + KBLK - 1) / KBLK - 1;
        if (__shfl_sync(FULL, last, 0)) {
            __threadfence();
            key_bases_warp(v, c, lane);
            if (lane == 0) v.kbdone[c] = 0;
        }
    }
}

// ---------------------------------------------------------------------------
// stable scatter: one warp per chunk walks its points in index order and
// writes each assigned point's coordinates to the next free row of its key's
// segment of the grouped copy Pg, so every segment lists its members in
// cloud-point index order as one contiguous stream for the folds.  Keys of the chunk and the per-key start slots are
// staged in shared memory first; the ordered walk then touches shared memory
// only (match_any groups equal keys of 32 consecutive points, the group
// leader advances the key's cursor).
// ---------------------------------------------------------------------------
template <int DIM>
__device__ void scatter_chunk(const EngineView& v, int c, int lc, int* s_keys, int lane);

// row r of a grouped copy (PadDim<DIM> floats per row)
template <int DIM>
__device__ __forceinline__ void store_row(float* rows, int64_t r, const float (&q)[DIM])
{
    constexpr int DP = PadDim<DIM>::v;
    if constexpr (DP == 4) {
        reinterpret_cast<float4*>(rows)[r] =
            make_float4(q[0], DIM > 1 ? q[DIM > 1 ? 1 : 0] : 0.0f, DIM > 2 ? q[DIM > 2 ? 2 : 0] : 0.0f,
                        DIM > 3 ? q[DIM > 3 ? 3 : 0] : 0.0f);
    } else if constexpr (DP == 2) {
        reinterpret_cast<float2*>(rows)[r] = make_float2(q[0], q[1]);
    } else {
#pragma unroll
        for (int d = 0; d < DIM; ++d) rows[r * DP + d] = q[d];
    }
}


// One CTA per chunk for clouds with at most SCAT_HMAX chosen points.  The
// chunk is split into SCAT_W contiguous warp ranges; every warp counts its
// range's keys, an exclusive scan over the warps (per key) gives every warp
// its own start slots, and the warps then place their ranges at the same time,
// each in index order.  Ranges are in index order too, so the placement stays
// stable while the dependent placement chain is SCAT_W times shorter.  Larger
// chosen sets use scatter_chunk (one warp) in warp 0.
// groups of more clouds than this are gathered and compacted one thread per
// cloud (decimate_group)
constexpr int DEC_CLOUDS_SERIAL = 32;
constexpr int SCAT_W = 8;
constexpr int SCAT_HMAX = 1024;
constexpr int SCAT_KS = 8;   // chunk keys per thread loaded together (covers 2,048-point chunks)
constexpr int SCAT_SP = 8;   // placement steps whose coordinates are loaded together
static_assert(SCAT_HMAX % (SCAT_W * 32) == 0, "key bases: whole loads per thread");

template <int DIM>
__global__ void __launch_bounds__(SCAT_W * 32) k_scatter_cta(EngineView v)
{
    pdl_enter();
    constexpr int DP = PadDim<DIM>::v;
    extern __shared__ int s_dyn[];
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const ActiveList al(v, ACT_CHUNK);
    for (int item = blockIdx.x; item < al.total; item += gridDim.x) {
        __syncthreads();  // the previous chunk's readers are done
        int c, lc;
        al.locate(item, c, lc);
        const CloudDesc cd = v.cl[c];
        const int ns = v.ns[c];
        if (ns > SCAT_HMAX) {
            if (warp == 0) scatter_chunk<DIM>(v, c, lc, s_dyn, lane);
            continue;
        }
        const int start = (int)(((int64_t)lc * cd.n_all) / cd.n_chunks);
        const int end = (int)(((int64_t)(lc + 1) * cd.n_all) / cd.n_chunks);
        const int len = end - start;
        int* s_keys = s_dyn;                 // chunk_max
        int* hw = s_dyn + v.chunk_max;       // SCAT_W x ns: counts, then start slots
        const int32_t* keys = v.keys + cd.p_off + start;
        int32_t* row = v.hist + cd.hist_off + (int64_t)lc * cd.ns_cap;
        const int32_t* bs = v.base + cd.key_off;
        const float* Pc = v.P + (cd.p_off + start) * DIM;
        const int r0 = (warp * len) / SCAT_W, r1 = ((warp + 1) * len) / SCAT_W;
        // Every global load of the chunk is issued up front -- its keys, its
        // key bases and histogram row, and the coordinates of this warp's
        // first SCAT_SP placement steps -- so the chunk waits for one memory
        // round trip instead of one per loop step.
        int kv[SCAT_KS];
#pragma unroll
        for (int u = 0; u < SCAT_KS; ++u) {
            const int e = u * SCAT_W * 32 + tid;
            kv[u] = (e < len) ? keys[e] : -1;
        }
        int bsv[SCAT_HMAX / (SCAT_W * 32)], rwv[SCAT_HMAX / (SCAT_W * 32)];
#pragma unroll
        for (int u = 0; u < SCAT_HMAX / (SCAT_W * 32); ++u) {
            const int k = u * SCAT_W * 32 + tid;
            bsv[u] = (k < ns) ? bs[k] : 0;
            rwv[u] = (k < ns) ? row[k] : 0;
        }
        float pc[SCAT_SP][DIM];
#pragma unroll
        for (int q = 0; q < SCAT_SP; ++q) {
            const int i = r0 + q * 32 + lane;
#pragma unroll
            for (int d = 0; d < DIM; ++d) pc[q][d] = (i < r1) ? Pc[(int64_t)i * DIM + d] : 0.0f;
        }
#pragma unroll
        for (int u = 0; u < SCAT_KS; ++u) {
            const int e = u * SCAT_W * 32 + tid;
            if (e < len) s_keys[e] = kv[u];
        }
        for (int e = SCAT_KS * SCAT_W * 32 + tid; e < len; e += SCAT_W * 32) s_keys[e] = keys[e];
        for (int e = tid; e < SCAT_W * ns; e += SCAT_W * 32) hw[e] = 0;
        __syncthreads();
        // per-warp key counts (order-free: shared-memory adds into the
        // warp's own row)
        for (int i = r0 + lane; i < r1; i += 32) {
            const int key = s_keys[i];
            if (key >= 0) atomicAdd(&hw[warp * ns + key], 1);
        }
        __syncthreads();
#pragma unroll
        for (int u = 0; u < SCAT_HMAX / (SCAT_W * 32); ++u) {
            const int k = u * SCAT_W * 32 + tid;
            if (k < ns) {
                int run = bsv[u] + rwv[u];
                row[k] = 0;  // the row is free again for the next pass's counts
#pragma unroll
                for (int w = 0; w < SCAT_W; ++w) {
                    const int x = hw[w * ns + k];
                    hw[w * ns + k] = run;
                    run += x;
                }
            }
        }
        __syncthreads();
        int* cur = hw + warp * ns;
        float* Pg = v.Pg + cd.p_off * DP;
        for (int g0 = r0; g0 < r1; g0 += 32 * SCAT_SP) {
            if (g0 > r0) {  // ranges longer than SCAT_SP steps: the next steps' coordinates
#pragma unroll
                for (int q = 0; q < SCAT_SP; ++q) {
                    const int i = g0 + q * 32 + lane;
#pragma unroll
                    for (int d = 0; d < DIM; ++d) pc[q][d] = (i < r1) ? Pc[(int64_t)i * DIM + d] : 0.0f;
                }
            }
#pragma unroll
            for (int q = 0; q < SCAT_SP; ++q) {
                const int i0 = g0 + q * 32;
                if (i0 >= r1) break;
                const int i = i0 + lane;
                const WarpRun r = warp_runs((i < r1) ? s_keys[i] : -1, lane);
                int b = 0;
                if (r.key >= 0 && lane == r.head) {
                    b = cur[r.key];
                    cur[r.key] = b + r.count;
                }
                b = __shfl_sync(FULL, b, r.head);
                float qv[DIM];
#pragma unroll
                for (int d = 0; d < DIM; ++d) qv[d] = __shfl_sync(FULL, pc[q][d], r.src);
                if (r.key >= 0) store_row<DIM>(Pg, b + r.rank, qv);
            }
        }
    }
}

// dynamic shared memory of k_scatter_cta
inline int scatter_cta_smem_bytes(const EngineView& v)
{
    const int block_path = v.chunk_max + SCAT_W * SCAT_HMAX;
    const int warp_path = v.chunk_max + v.scat_smem;
    return 4 * (block_path > warp_path ? block_path : warp_path);
}

template <int DIM>
__device__ void scatter_chunk(const EngineView& v, int c, int lc, int* s_keys, int lane)
{
    constexpr int DP = PadDim<DIM>::v;
    const CloudDesc cd = v.cl[c];
    const int ns = v.ns[c];
    int32_t* row = v.hist + cd.hist_off + (int64_t)lc * cd.ns_cap;
    const int32_t* bs = v.base + cd.key_off;
    const bool in_smem = ns <= v.scat_smem;
    int32_t* ctr = in_smem ? (s_keys + v.chunk_max) : row;
    const int start = (int)(((int64_t)lc * cd.n_all) / cd.n_chunks);
    const int end = (int)(((int64_t)(lc + 1) * cd.n_all) / cd.n_chunks);
    const int len = end - start;
    const int32_t* keys = v.keys + cd.p_off + start;
    // stage the chunk's keys and the per-key start slots: eight independent
    // loads per lane in flight before the first shared-memory store, so the
    // staging costs a few load latencies instead of one per 32 elements
    for (int e0 = 0; e0 < len; e0 += 32 * 8) {
        int t[8];
#pragma unroll
        for (int u = 0; u < 8; ++u) {
            const int e = e0 + u * 32 + lane;
            t[u] = (e < len) ? keys[e] : 0;
        }
#pragma unroll
        for (int u = 0; u < 8; ++u) {
            const int e = e0 + u * 32 + lane;
            if (e < len) s_keys[e] = t[u];
        }
    }
    for (int k0 = 0; k0 < ns; k0 += 32 * 4) {
        int a[4], r[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const int k = k0 + u * 32 + lane;
            a[u] = (k < ns) ? bs[k] : 0;
            r[u] = (k < ns) ? row[k] : 0;
        }
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const int k = k0 + u * 32 + lane;
            if (k < ns) ctr[k] = a[u] + r[u];
        }
    }
    __syncwarp();
    const float* Pc = v.P + (cd.p_off + start) * DIM;
    float* Pg = v.Pg + cd.p_off * DP;
    for (int off = 0; off < len; off += 32) {
        const int i = off + lane;
        float pc[DIM];
#pragma unroll
        for (int d = 0; d < DIM; ++d) pc[d] = (i < len) ? Pc[(int64_t)i * DIM + d] : 0.0f;
        const WarpRun r = warp_runs((i < len) ? s_keys[i] : -1, lane);
        int b = 0;
        if (r.key >= 0 && lane == r.head) {
            b = ctr[r.key];
            ctr[r.key] = b + r.count;
        }
        b = __shfl_sync(FULL, b, r.head);
        float q[DIM];
#pragma unroll
        for (int d = 0; d < DIM; ++d) q[d] = __shfl_sync(FULL, pc[d], r.src);
        if (r.key >= 0) store_row<DIM>(Pg, b + r.rank, q);
        __syncwarp();
    }
    for (int k = lane; k < ns; k += 32) row[k] = 0;  // free for the next pass's counts
}

// ---------------------------------------------------------------------------
// ordered sum + shift: one warp per chosen slot.  Lane d (< DIM) folds
// coordinate d of the key's members in index order with rounded adds,
// exactly as rd/cpu/brute_force/evolve.hpp:71-74 accumulates, then applies the
// movement test of evolve.hpp:143-177.  Members are gathered through the
// permutation written by k_scatter_cta, BP at a time, the next block in flight
// while the current one is folded.
// ---------------------------------------------------------------------------
constexpr int SUM_BP = 128;  // members staged per step of the ordered fold
// k_sum_shift stages 256 members per step: folding a block (about 256 dependent
// adds) then outlasts the gather of the next one from L2
constexpr int SUM_BP_WIDE = 256;
// points (keys) per lane loaded together by the fused tile kernel's
// assignment (placement) loop
constexpr int TILE_PPL = 8;
// members from which the fused tile kernel folds a key with the whole CTA
// (warp-segmented exact evaluation, rd_segfold.cuh) instead of one warp's add
// chain
constexpr int FOLD_CTA_MIN = 4096;
// the same for the light tiles of the cluster kernel: the heavy tiles, whose
// keys need the CTA-wide folds, went to clusters; the others fold faster with
// every warp on its own keys
constexpr int FOLD_CTA_MIN_LIGHT = 1 << 30;

template <int DIM>
__device__ void sum_shift_one(const EngineView& v, int c, int k, float* buf, int lane, bool cta_big);

template <int DIM>
__device__ void sum_shift_big_one(const EngineView& v, int slot, SegFoldSmem<8, DIM>& sm);

// the per-cloud control step after a pass (k_control), over clouds first,
// first + stride, ... of the active list
__device__ void control_clouds(const EngineView& v, const int first, const int stride);

// grid = big_ctas CTAs for the listed big keys (one key at a time each), then
// the CTAs whose warps take one smaller key each
// with_control: the last CTA to finish runs the control step of k_control
// (the moved flags of every fold are then complete)
template <int DIM>
__global__ void __launch_bounds__(256) k_sum_shift(EngineView v, int big_ctas, int with_control)
{
    pdl_enter();
    __shared__ __align__(16) unsigned char s_raw[8 * SUM_BP_WIDE * (DIM + 1) * 4];
    __shared__ int s_last;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int nbig = v.ctr[CTR_NBIG];
    const bool cta_big = nbig <= SUM_BIG_PER_CTA * big_ctas;  // else every key goes to a warp
    if ((int)blockIdx.x < big_ctas) {
        static_assert(sizeof(SegFoldSmem<8, DIM>) <= sizeof(s_raw), "big-key fold scratch");
        SegFoldSmem<8, DIM>& sm = *reinterpret_cast<SegFoldSmem<8, DIM>*>(s_raw);
        if (cta_big)
            for (int i = blockIdx.x; i < nbig; i += big_ctas) sum_shift_big_one<DIM>(v, v.big[i], sm);
    } else {
        float* s_buf = reinterpret_cast<float*>(s_raw) + warp * SUM_BP_WIDE * PadDim<DIM>::v;
        const ActiveList al(v, ACT_SLOT);
        const int b = (int)blockIdx.x - big_ctas, nb = (int)gridDim.x - big_ctas;
        for (int t = b * 8 + warp; t < al.total; t += nb * 8) {
            __syncwarp();
            int c, k;
            al.locate(t, c, k);
            sum_shift_one<DIM>(v, c, k, s_buf, lane, cta_big);
        }
    }
    if (!with_control) return;
    // every thread's writes (chosen points, moved flags) before the count
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) s_last = atomicAdd(&v.ctr[CTR_SUM_DONE], 1) == (int)gridDim.x - 1;
    __syncthreads();
    if (!s_last) return;
    __threadfence();
    control_clouds(v, threadIdx.x, blockDim.x);
    if (threadIdx.x == 0) v.ctr[CTR_SUM_DONE] = 0;
}

// Sequential FP32 fold, in list order, of the points P[perm[0..n)] (one warp;
// the sum of coordinate d is returned in lane d < DIM).
template <int DIM, int BP = SUM_BP>
__device__ float fold_members(const int32_t* __restrict__ perm, const int n,
                              const float* __restrict__ P, float* buf, int* sidx, const int lane)
{
    constexpr int R = BP * DIM / 32;    // floats per lane per step
    float nxt[R];
    // Two-stage pipeline: member indices of block b+2 and coordinates of
    // block b+1 are in flight while block b is folded.
    int pnx[BP / 32];
    auto load_perm = [&](int off) {
        const int m = min(BP, n - off);
#pragma unroll
        for (int u = 0; u < BP / 32; ++u) {
            const int j = u * 32 + lane;
            pnx[u] = (off < n && j < m) ? perm[off + j] : 0;
        }
    };
    auto load_coords = [&](int off) {  // indices of block `off` are in sidx
        const int m = min(BP, n - off);
#pragma unroll
        for (int u = 0; u < R; ++u) {
            const int e = u * 32 + lane;
            const int j = e / DIM, d = e - (e / DIM) * DIM;
            nxt[u] = (j < m) ? P[(int64_t)sidx[j] * DIM + d] : 0.0f;
        }
    };
    auto stage_perm = [&]() {
#pragma unroll
        for (int u = 0; u < BP / 32; ++u) sidx[u * 32 + lane] = pnx[u];
        __syncwarp();
    };
    load_perm(0);
    stage_perm();
    load_coords(0);
    load_perm(BP);
    float sum = 0.0f;
    for (int off = 0; off < n; off += BP) {
        const int m = min(BP, n - off);
        __syncwarp();  // every lane is done reading sidx of the previous stage
#pragma unroll
        for (int u = 0; u < R; ++u) buf[u * 32 + lane] = nxt[u];
        if (off + BP < n) {
            stage_perm();               // indices of block off+BP
            load_coords(off + BP);      // in flight during the fold
            load_perm(off + 2 * BP);    // in flight during the fold
        }
        __syncwarp();
        if (lane < DIM) {
            if (m == BP) {
#pragma unroll 32
                for (int j = 0; j < BP; ++j) sum = __fadd_rn(sum, buf[j * DIM + lane]);
            } else {
                for (int j = 0; j < m; ++j) sum = __fadd_rn(sum, buf[j * DIM + lane]);
            }
        }
        __syncwarp();
    }
    return sum;
}

// The shift of chosen point k of cloud c from its members' sum (lane d < DIM
// holds coordinate d): evolve.hpp:143-177, or the plain mean for the
// adjoint's forward step.  Called by one whole warp.
template <int DIM>
__device__ void apply_shift(const EngineView& v, int c, const CloudDesc& cd, int k, int n, float sum,
                            int lane)
{
    int moved = 0;
    if (lane < DIM) {
        float* s = v.S + (cd.s_off + k) * DIM + lane;
        if (v.flags & ENG_ALWAYS_MOVE) {
            *s = __fdiv_rn(sum, (float)n);  // mean, no movement test
        } else {
            float cval = *s;
            moved = shift_coord(sum, n, cval);
            if (moved) *s = cval;
        }
    }
    if (__any_sync(FULL, moved) && lane == 0) v.cont[c] = 1;
}

// Sequential FP32 fold, in order, of n contiguous rows of a grouped copy
// (PadDim<DIM> floats each); one warp, the sum of coordinate d returned in
// lane d < DIM.  A block of BP rows is loaded with coalesced vector loads into
// the warp's buffer (BP x PadDim floats) while the previous block is folded.
template <int DIM, int BP>
__device__ float fold_rows(const float* __restrict__ rows, const int n, float* buf, const int lane)
{
    constexpr int DP = PadDim<DIM>::v;
    constexpr int VW = (DP == 4) ? 4 : (DP == 2 ? 2 : 1);  // floats per vector load
    constexpr int R = BP * DP / (32 * VW);                 // vector loads per lane per block
    static_assert(BP * DP % (32 * VW) == 0, "block of whole vector loads");
    float nxt[R][VW];
    auto load = [&](int off) {
        const int lim = min(BP, n - off) * DP;  // valid floats of the block
        const float* src = rows + (int64_t)off * DP;
#pragma unroll
        for (int u = 0; u < R; ++u) {
            const int e = (u * 32 + lane) * VW;
            if constexpr (VW == 4) {
                const float4 t = (e < lim) ? reinterpret_cast<const float4*>(src)[u * 32 + lane]
                                           : make_float4(0.f, 0.f, 0.f, 0.f);
                nxt[u][0] = t.x; nxt[u][VW > 1 ? 1 : 0] = t.y;
                nxt[u][VW > 2 ? 2 : 0] = t.z; nxt[u][VW > 3 ? 3 : 0] = t.w;
            } else if constexpr (VW == 2) {
                const float2 t = (e < lim) ? reinterpret_cast<const float2*>(src)[u * 32 + lane]
                                           : make_float2(0.f, 0.f);
                nxt[u][0] = t.x; nxt[u][VW > 1 ? 1 : 0] = t.y;
            } else {
                nxt[u][0] = (e < lim) ? src[e] : 0.0f;
            }
        }
    };
    load(0);
    float sum = 0.0f;
    for (int off = 0; off < n; off += BP) {
        const int m = min(BP, n - off);
        __syncwarp();  // every lane is done reading the previous block
#pragma unroll
        for (int u = 0; u < R; ++u)
#pragma unroll
            for (int w = 0; w < VW; ++w) buf[(u * 32 + lane) * VW + w] = nxt[u][w];
        if (off + BP < n) load(off + BP);  // in flight during the fold
        __syncwarp();
        if (lane < DIM) {
            if (m == BP) {
#pragma unroll 32
                for (int j = 0; j < BP; ++j) sum = __fadd_rn(sum, buf[j * DP + lane]);
            } else {
                for (int j = 0; j < m; ++j) sum = __fadd_rn(sum, buf[j * DP + lane]);
            }
        }
    }
    __syncwarp();
    return sum;
}

template <int DIM>
__device__ void sum_shift_one(const EngineView& v, int c, int k, float* buf, int lane, bool cta_big)
{
    const CloudDesc cd = v.cl[c];
    const int n = v.cnt[cd.key_off + k];
    if (n == 0 || (cta_big && n >= SUM_BIG_MIN)) return;  // big keys: the CTA path
    const float* rows = v.Pg + (cd.p_off + v.base[cd.key_off + k]) * PadDim<DIM>::v;
    const float sum = fold_rows<DIM, SUM_BP_WIDE>(rows, n, buf, lane);
    apply_shift<DIM>(v, c, cd, k, n, sum, lane);
}

// ---------------------------------------------------------------------------
// The same ordered sum + shift for one key of SUM_BIG_MIN or more members
// (global chosen slot `slot`), by a whole CTA: warps 1..7 gather the members'
// coordinates (in member order) into one of two shared buffers while warp 0
// folds the other with the same chain of rounded adds (lane d: coordinate
// d), so the gathers of a large cluster no longer stall its add chain.
// ---------------------------------------------------------------------------
// One big key folded by the whole CTA: the warp-segmented exact fold of
// rd_segfold.cuh (eight warp segments from speculative starts, traces replayed
// from the exact start), then the shift.
template <int DIM>
__device__ void sum_shift_big_one(const EngineView& v, int slot, SegFoldSmem<8, DIM>& sm)
{
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int c = v.slot_cloud[slot];
    const CloudDesc cd = v.cl[c];
    const int k = (int)(slot - cd.key_off);
    const int n = v.cnt[slot];
    const float* rows = v.Pg + (cd.p_off + v.base[slot]) * PadDim<DIM>::v;
    __syncthreads();  // the previous key's scratch is no longer read
    fold_members_seg_src<8, DIM>(RowSrc<DIM>{rows}, n, sm);
    if (warp == 0) apply_shift<DIM>(v, c, cd, k, n, (lane < DIM) ? sm.out[lane] : 0.0f, lane);
}

// ---------------------------------------------------------------------------
// Fused per-tile evolve (tiled runs): one CTA evolves one tile to convergence
// without leaving the kernel, so tiles proceed independently instead of in
// lockstep passes.  Every pass is the same exact computation as the pass
// pipeline (assign with the two-level argmin, stable grouping, index-order
// fold, movement test), done inside the CTA:
//   * warp w owns the contiguous point range [w n/W, (w+1) n/W); its per-key
//     counts go to hist[w][key];
//   * a key's members are laid out warp range by warp range, each range in
//     index order (match_any ranks inside 32-point steps), i.e. in index order;
//   * warp w folds keys w, w+W, ... (fold_members) and applies the shift.
// Shared memory: chosen points (TILE_NS_MAX, padded to float4 for DIM 3),
// W x (ns+1) counters, key bases.
// ---------------------------------------------------------------------------
// Assignment of the points [r0, r1w) of a tile by one warp (steps of 32 x
// TILE_PPL points, loads first): keys[i] = nearest chosen point within r1
// (first index of the minimum), and the warp's members per key in whist.
// With at most TILE_KB chosen points the counts are kept per key in
// warp-uniform registers (one ballot per key and step) and stored at the end;
// otherwise one shared-memory add per distinct key of a step.
constexpr int TILE_KB = 8;

template <int DIM>
__device__ __forceinline__ void tile_assign_range(const float* __restrict__ P, const int r0,
                                                  const int r1w, const float* sS, const int ns,
                                                  const int nsp, const float rsq,
                                                  int32_t* __restrict__ keys, int* whist,
                                                  const int lane)
{
    constexpr int KB = TILE_KB;
    int kc[KB];
#pragma unroll
    for (int k = 0; k < KB; ++k) kc[k] = 0;
    for (int i0 = r0; i0 < r1w; i0 += 32 * TILE_PPL) {
        float p[TILE_PPL][DIM];
#pragma unroll
        for (int h = 0; h < TILE_PPL; ++h) {
            const int i = i0 + h * 32 + lane;
#pragma unroll
            for (int d = 0; d < DIM; ++d) p[h][d] = (i < r1w) ? P[(int64_t)i * DIM + d] : 0.0f;
        }
        if (ns <= KB) {
            // first index of the minimum, directly: each chosen point is read
            // once for the step's TILE_PPL points
            float best[TILE_PPL];
            int bk[TILE_PPL];
#pragma unroll
            for (int h = 0; h < TILE_PPL; ++h) {
                best[h] = FLT_MAX;
                bk[h] = -1;
            }
            for (int k = 0; k < ns; ++k) {
                float s[DIM];
                load_chosen<DIM>(sS, k, s);
#pragma unroll
                for (int h = 0; h < TILE_PPL; ++h) {
                    const float dd = sqdist_exact<DIM>(s, p[h]);
                    if (dd < best[h]) { best[h] = dd; bk[h] = k; }
                }
            }
#pragma unroll
            for (int h = 0; h < TILE_PPL; ++h) {
                const int i = i0 + h * 32 + lane;
                const int key = (i < r1w && best[h] <= rsq) ? bk[h] : -1;
                if (i < r1w) keys[i] = key;
#pragma unroll
                for (int k = 0; k < KB; ++k)
                    if (k < ns) kc[k] += __popc(__ballot_sync(FULL, key == k));
            }
            continue;
        }
#pragma unroll
        for (int h = 0; h < TILE_PPL; ++h) {
            const int i = i0 + h * 32 + lane;
            int key = -1;
            if (i < r1w) {
                float best = FLT_MAX;
                int blk = -1;
                for (int kb = 0; kb < nsp; kb += KB) {
                    const float old = best;
#pragma unroll
                    for (int u = 0; u < KB; ++u) {
                        float s[DIM];
                        load_chosen<DIM>(sS, kb + u, s);
                        best = fminf(best, sqdist_exact<DIM>(s, p[h]));
                    }
                    blk = (best < old) ? kb : blk;
                }
                if (best <= rsq && blk >= 0) {
                    for (int u = 0; u < KB && blk + u < ns; ++u) {
                        float s[DIM];
                        load_chosen<DIM>(sS, blk + u, s);
                        if (sqdist_exact<DIM>(s, p[h]) == best) { key = blk + u; break; }
                    }
                }
                keys[i] = key;
            }
            // a tile's warp step holds few distinct keys: the match
            // instruction is cheap there (warp_runs suits many keys)
            const unsigned mm = __match_any_sync(FULL, key);
            if (key >= 0 && lane == __ffs(mm) - 1) atomicAdd(&whist[key], __popc(mm));
        }
    }
    if (ns <= KB && lane == 0)
#pragma unroll
        for (int k = 0; k < KB; ++k)
            if (k < ns) whist[k] += kc[k];
}

// Stable placement of the warp's points [r0, r1w): the coordinates of the
// members of key k go, in index order, to rows cur[k], cur[k] + 1, ... of the
// grouped copy Pg (cur advanced).
template <int DIM>
__device__ __forceinline__ void tile_place_range(const float* __restrict__ P,
                                                 const int32_t* __restrict__ keys, const int r0,
                                                 const int r1w, int* cur, const int ns,
                                                 float* __restrict__ Pg, const int lane)
{
    constexpr int KB = TILE_KB;
    int base[KB];
    if (ns <= KB) {
#pragma unroll
        for (int k = 0; k < KB; ++k) base[k] = (k < ns) ? cur[k] : 0;
    }
    for (int i0 = r0; i0 < r1w; i0 += 32 * TILE_PPL) {
        int kq[TILE_PPL];
        float pq[TILE_PPL][DIM];
#pragma unroll
        for (int h = 0; h < TILE_PPL; ++h) {
            const int i = i0 + h * 32 + lane;
            kq[h] = (i < r1w) ? keys[i] : -1;
#pragma unroll
            for (int d = 0; d < DIM; ++d) pq[h][d] = (i < r1w) ? P[(int64_t)i * DIM + d] : 0.0f;
        }
#pragma unroll
        for (int h = 0; h < TILE_PPL; ++h) {
            const int key = kq[h];
            if (ns <= KB) {
#pragma unroll
                for (int k = 0; k < KB; ++k) {
                    if (k < ns) {
                        const unsigned m = __ballot_sync(FULL, key == k);
                        if (key == k) store_row<DIM>(Pg, base[k] + __popc(m & lanemask_lt()), pq[h]);
                        base[k] += __popc(m);
                    }
                }
            } else {
                const unsigned m = __match_any_sync(FULL, key);
                const int leader = __ffs(m) - 1;
                int b = 0;
                if (key >= 0 && lane == leader) {
                    b = cur[key];
                    cur[key] = b + __popc(m);
                }
                b = __shfl_sync(FULL, b, leader);
                if (key >= 0) store_row<DIM>(Pg, b + __popc(m & lanemask_lt()), pq[h]);
            }
        }
    }
}

template <int DIM, int BLOCK>
struct TileCtaSmem {
    float buf[BLOCK / 32][SUM_BP * PadDim<DIM>::v];   // fold_rows blocks
    int moved;
    SegFoldSmem<BLOCK / 32, DIM> seg;
};

// One CTA evolves tile c to convergence (see above); dyn is the dynamic
// shared memory laid out as tile_evolve_smem_bytes describes.
template <int DIM, int BLOCK>
__device__ void tile_evolve_one(const EngineView& v, const int c, const int fold_cta_min,
                                unsigned char* dyn,
                                TileCtaSmem<DIM, BLOCK>& ts)
{
    constexpr int W = BLOCK / 32;
    constexpr int DP = PadDim<DIM>::v;
    constexpr int KB = 8;
    constexpr float FAR = 1e30f;
    float* sS = reinterpret_cast<float*>(dyn);                              // TILE_NS_MAX*DP
    int* hist = reinterpret_cast<int*>(sS + TILE_NS_MAX * DP);             // W*(TILE_NS_MAX+1)
    int* kbase = hist + W * (TILE_NS_MAX + 1);                              // TILE_NS_MAX+1
    auto& s_buf = ts.buf;
    int& s_moved = ts.moved;
    auto& s_seg = ts.seg;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    {
        const CloudDesc cd = v.cl[c];
        const int n = cd.n_all;
        const int ns = v.ns[c];
        const float* P = v.P + cd.p_off * DIM;
        float* gS = v.S + cd.s_off * DIM;
        int32_t* keys = v.keys + cd.p_off;
        float* Pg = v.Pg + cd.p_off * DP;
        const float rsq = sqr_rn(cd.r1);
        const int nsp = (ns + KB - 1) / KB * KB;
        __syncthreads();
        for (int e = tid; e < nsp; e += BLOCK)
#pragma unroll
            for (int d = 0; d < DIM; ++d) sS[e * DP + d] = (e < ns) ? gS[(int64_t)e * DIM + d] : FAR;
        const int r0 = (int)(((int64_t)warp * n) / W), r1w = (int)(((int64_t)(warp + 1) * n) / W);
        int pass = 0;
        for (;;) {
            // 1. assignment of the warp's range + per-warp key counts
            //    (counts added once per distinct key of a warp step)
            for (int k = lane; k <= ns; k += 32) hist[warp * (TILE_NS_MAX + 1) + k] = 0;
            __syncthreads();
            int* whist = hist + warp * (TILE_NS_MAX + 1);
            tile_assign_range<DIM>(P, r0, r1w, sS, ns, nsp, rsq, keys, whist, lane);
            __syncthreads();
            // 2. key bases and per-warp starts (thread per key)
            for (int k = tid; k < ns; k += BLOCK) {
                int tot = 0;
                for (int w = 0; w < W; ++w) tot += hist[w * (TILE_NS_MAX + 1) + k];
                kbase[k + 1] = tot;  // counts for the scan below
            }
            if (tid == 0) { kbase[0] = 0; s_moved = 0; }
            __syncthreads();
            if (warp == 0) {  // inclusive scan of counts -> kbase[k] = first slot of key k
                int carry = 0;
                for (int k0 = 0; k0 < ns; k0 += 32) {
                    const int k = k0 + lane;
                    const int x = (k < ns) ? kbase[k + 1] : 0;
                    int incl = x;
#pragma unroll
                    for (int o = 1; o < 32; o <<= 1) {
                        const int y = __shfl_up_sync(FULL, incl, o);
                        if (lane >= o) incl += y;
                    }
                    if (k < ns) kbase[k + 1] = carry + incl;
                    carry += __shfl_sync(FULL, incl, 31);
                }
            }
            __syncthreads();
            for (int k = tid; k < ns; k += BLOCK) {
                int run = kbase[k];
                for (int w = 0; w < W; ++w) {
                    const int x = hist[w * (TILE_NS_MAX + 1) + k];
                    hist[w * (TILE_NS_MAX + 1) + k] = run;
                    run += x;
                }
            }
            __syncthreads();
            // 3. stable placement, warp range by warp range (keys of
            //    TILE_PPL warp steps loaded ahead of the dependent placement
            //    chain)
            tile_place_range<DIM>(P, keys, r0, r1w, hist + warp * (TILE_NS_MAX + 1), ns, Pg, lane);
            __syncthreads();
            // 4a. very large keys, one at a time, folded by the whole CTA
            for (int k = 0; k < ns; ++k) {
                const int cnt = kbase[k + 1] - kbase[k];
                if (cnt < fold_cta_min) continue;
                fold_members_seg_src<W, DIM>(RowSrc<DIM>{Pg + (int64_t)kbase[k] * DP}, cnt, s_seg);
                if (tid < DIM) {
                    float cval = sS[k * DP + tid];
                    if (shift_coord(s_seg.out[tid], cnt, cval)) {
                        sS[k * DP + tid] = cval;
                        s_moved = 1;
                    }
                }
                __syncthreads();
            }
            // 4b. index-order fold and movement test, warp w takes keys w, w+W, ...
            for (int k = warp; k < ns; k += W) {
                const int cnt = kbase[k + 1] - kbase[k];
                if (cnt == 0 || cnt >= fold_cta_min) continue;
                const float sum = fold_rows<DIM, SUM_BP>(Pg + (int64_t)kbase[k] * DP, cnt, s_buf[warp], lane);
                int moved = 0;
                if (lane < DIM) {
                    float cval = sS[k * DP + lane];
                    moved = shift_coord(sum, cnt, cval);
                    if (moved) sS[k * DP + lane] = cval;
                }
                if (__any_sync(FULL, moved) && lane == 0) s_moved = 1;
            }
            __syncthreads();
            ++pass;
            if (tid == 0) {
                v.pairs[c] += (unsigned long long)n * (unsigned long long)ns;
            }
            if (!s_moved) break;
            if (pass >= v.max_passes) {
                if (tid == 0) v.err[c] |= ERRB_EVOLVE_CAP;
                break;
            }
        }
        // results back and control (as k_control does after the last pass)
        for (int e = tid; e < ns; e += BLOCK)
#pragma unroll
            for (int d = 0; d < DIM; ++d) gS[(int64_t)e * DIM + d] = sS[e * DP + d];
        if (tid == 0) {
            v.passes[c] += pass;
            v.total_passes[c] += pass;
            v.cont[c] = 0;
            v.phase[c] = PH_CONVERGED;
            const GroupDesc gd = v.gr[cd.group];
            if (atomicAdd(&v.group_conv[cd.group], 1) + 1 == gd.n_clouds)
                v.ready[atomicAdd(&v.ctr[CTR_NREADY], 1)] = cd.group;
        }
    }
}

template <int DIM, int BLOCK>
__global__ void __launch_bounds__(BLOCK) k_tile_evolve(EngineView v)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ TileCtaSmem<DIM, BLOCK> ts;
    const int nact = v.ctr[CTR_NACT];
    for (int a = blockIdx.x; a < nact; a += gridDim.x)
        tile_evolve_one<DIM, BLOCK>(v, v.act_cloud[a], FOLD_CTA_MIN, smem_raw, ts);
}

__host__ __device__ constexpr int tile_evolve_smem_bytes(int dim)
{
    const int dp = (dim == 3) ? 4 : dim;
    const int w = 8;
    return TILE_NS_MAX * dp * 4 + w * (TILE_NS_MAX + 1) * 4 + (TILE_NS_MAX + 1) * 4;
}

}  // namespace
}  // namespace rdb
#include "rd_tile_cluster.cuh"
namespace rdb {
namespace {

// ---------------------------------------------------------------------------
// control: one thread per cloud after each pass.
// ---------------------------------------------------------------------------
__device__ void control_clouds(const EngineView& v, const int first, const int stride)
{
    const int nact = v.ctr[CTR_NACT];
    for (int a = first; a < nact; a += stride) {
        const int c = v.act_cloud[a];
        const CloudDesc cd = v.cl[c];
        v.pairs[c] += (unsigned long long)cd.n_all * (unsigned long long)v.ns[c];
        v.passes[c] += 1;
        v.total_passes[c] += 1;
        bool conv = false;
        if (v.cont[c] == 0) {
            conv = true;
        } else if (v.passes[c] >= v.max_passes) {
            v.err[c] |= ERRB_EVOLVE_CAP;
            conv = true;
        }
        v.cont[c] = 0;
        if (conv && (v.flags & ENG_EVOLVE_ONLY)) {
            v.phase[c] = PH_DONE;
        } else if (conv) {
            v.phase[c] = PH_CONVERGED;
            // the last member of a group to converge queues the group
            const GroupDesc gd = v.gr[cd.group];
            if (atomicAdd(&v.group_conv[cd.group], 1) + 1 == gd.n_clouds)
                v.ready[atomicAdd(&v.ctr[CTR_NREADY], 1)] = cd.group;
        }
    }
}

__global__ void k_control(EngineView v)
{
    pdl_enter();
    control_clouds(v, blockIdx.x * blockDim.x + threadIdx.x, gridDim.x * blockDim.x);
}

// ---------------------------------------------------------------------------
// decimate: one CTA per group, rd/cpu/brute_force/decimate.hpp:41-81 (brute
// force) or :85-127 (decimateNoCopy, tiled), on the group's chosen points in
// cloud order.  Neighbour counts within r2 and 2*r2 (self included) come from a
// hashed grid of cell edge > 2*r2; the in-order scan is kept exact by updating
// the counts of a removed point's neighbours at the moment of its removal, and
// a warp ballot skips runs of points that cannot be removed.
// ---------------------------------------------------------------------------
template <int DIM, int BLOCK>
__device__ void decimate_group(const EngineView& v, const int g)
{
    const GroupDesc gd = v.gr[g];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    __shared__ int s_off[33];
    __syncthreads();

    const CloudDesc c0 = v.cl[gd.cloud_begin];
    float* X = v.dx + gd.s_scratch * DIM;
    int32_t* cell = v.dcell + gd.s_scratch * DIM;
    int32_t* alive = v.dalive + gd.s_scratch;
    int32_t* c1 = v.dc1 + gd.s_scratch;
    int32_t* c2 = v.dc2 + gd.s_scratch;
    int32_t* items = v.ditems + gd.s_scratch;
    const int hbits = v.dec_hbits[g];
    const uint32_t hmask = (1u << hbits) - 1;
    int32_t* bstart = v.dbstart + v.dec_hoff[g];

    // Groups of many clouds (tiled runs) are walked one thread per cloud: the
    // clouds' offsets in the group's list come from a block-wide scan of their
    // chosen counts, or from the GPU-wide preparation (dcpre) when it ran.
    const int prepared = (v.dbig[0] == 1 && v.dbig[1] == g) ? 1 : 0;
    const bool per_thread = gd.n_clouds > DEC_CLOUDS_SERIAL;
    // f(ci, c, ns, off) for every cloud of the group, one thread each; returns
    // the group's total (the same in every thread)
    auto for_clouds = [&](auto&& f) -> int {
        __shared__ int s_w[BLOCK / 32];
        __shared__ int s_carry;
        if (tid == 0) s_carry = 0;
        __syncthreads();
        for (int c0 = 0; c0 < gd.n_clouds; c0 += BLOCK) {
            const int ci = c0 + tid;
            const int c = gd.cloud_begin + ci;
            const int x = (ci < gd.n_clouds) ? v.ns[c] : 0;
            int incl = x;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const int y = __shfl_up_sync(FULL, incl, o);
                if (lane >= o) incl += y;
            }
            if (lane == 31) s_w[warp] = incl;
            __syncthreads();
            int pre = 0, tot = 0;
            for (int w = 0; w < BLOCK / 32; ++w) {
                pre += (w < warp) ? s_w[w] : 0;
                tot += s_w[w];
            }
            const int carry = s_carry;
            if (ci < gd.n_clouds) f(ci, c, x, prepared ? v.dcpre[ci] : carry + pre + incl - x);
            __syncthreads();
            if (tid == 0) s_carry = carry + tot;
            __syncthreads();
        }
        return s_carry;
    };
    // gather the group's chosen points (cloud order) into X, unless the
    // GPU-wide preparation kernels already did (large group)
    int total = 0;
    if (prepared) {
        total = v.dbig[2];
    } else if (per_thread) {
        total = for_clouds([&](int, int c, int ns, int off) {
            const int64_t so = v.cl[c].s_off;
            for (int e = 0; e < ns * DIM; ++e) X[(int64_t)off * DIM + e] = v.S[so * DIM + e];
        });
        __syncthreads();
    } else {
        for (int i = 0; i < gd.n_clouds; ++i) {
            const int c = gd.cloud_begin + i;
            const CloudDesc cd = v.cl[c];
            const int ns = v.ns[c];
            for (int e = tid; e < ns * DIM; e += BLOCK) X[(int64_t)total * DIM + e] = v.S[cd.s_off * DIM + e];
            total += ns;
        }
    }
    extern __shared__ __align__(16) unsigned char dec_smem[];
    decimate_scan_lists<DIM, BLOCK>(X, total, c0.r2, gd.nocopy, cell, alive, c1, c2, items, bstart,
                                    hmask, v.dnb_off + gd.s_scratch + g,
                                    v.dnb + (int64_t)v.dec_nb_pp * gd.s_scratch,
                                    (int64_t)v.dec_nb_pp * gd.s_cap, dec_smem, v.dec_smem_max,
                                    &v.err[gd.cloud_begin], prepared, v.ctr + CTR_DEC_PASSES);
    // compaction back into each cloud, in order
    int running = 0, total_after = 0;
    if (per_thread) {
        __shared__ int s_after;
        if (tid == 0) s_after = 0;
        __syncthreads();
        int mine = 0;
        for_clouds([&](int, int c, int ns, int off) {
            const int64_t so = v.cl[c].s_off;
            int kept = 0;
            for (int k = 0; k < ns; ++k) {
                if (!alive[off + k]) continue;
#pragma unroll
                for (int d = 0; d < DIM; ++d) v.S[(so + kept) * DIM + d] = X[(int64_t)(off + k) * DIM + d];
                ++kept;
            }
            v.ns[c] = kept;
            mine += kept;
        });
        if (mine) atomicAdd(&s_after, mine);
        __syncthreads();
        total_after = s_after;
    }
    for (int ci = 0; !per_thread && ci < gd.n_clouds; ++ci) {
        const int c = gd.cloud_begin + ci;
        const CloudDesc cd = v.cl[c];
        const int ns = v.ns[c];
        int kept = 0;
        for (int k0 = 0; k0 < ns; k0 += BLOCK) {
            const int k = k0 + tid;
            const bool a = (k < ns) && alive[running + k];
            const unsigned bal = __ballot_sync(FULL, a);
            if (lane == 0) s_off[warp] = __popc(bal);
            __syncthreads();
            int pre = 0, tot = 0;
            for (int w = 0; w < BLOCK / 32; ++w) {
                pre += (w < warp) ? s_off[w] : 0;
                tot += s_off[w];
            }
            if (a) {
                const int pos = kept + pre + __popc(bal & lanemask_lt());
#pragma unroll
                for (int d = 0; d < DIM; ++d)
                    v.S[(cd.s_off + pos) * DIM + d] = X[(int64_t)(running + k) * DIM + d];
            }
            kept += tot;
            __syncthreads();
        }
        running += ns;
        total_after += kept;
        if (tid == 0) v.ns[c] = kept;
    }
    __syncthreads();
    // outer-loop control: stop when decimation removed nothing
    const bool stable = (total_after == total);
    for (int i = tid; i < gd.n_clouds; i += BLOCK) {
        const int c = gd.cloud_begin + i;
        v.outer[c] += 1;
        v.passes[c] = 0;
        if (stable) {
            v.phase[c] = PH_DONE;
        } else if (v.outer[c] >= v.max_outer) {
            v.err[c] |= ERRB_OUTER_CAP;
            v.phase[c] = PH_DONE;
        } else {
            v.phase[c] = PH_EVOLVE;
        }
    }
    if (tid == 0) {
        v.group_conv[g] = 0;
        if (prepared) v.dbig[0] = 0;
    }
    __syncthreads();
}

// ---------------------------------------------------------------------------
// GPU-wide preparation of a large decimation (tiled runs: one group of
// thousands of tiles).  When exactly one group is ready and it holds more
// than DEC_BIG_MIN points, these kernels build its gathered points, hash
// buckets, neighbour counts and neighbour lists across all SMs; k_decimate
// then only runs the in-order scan.  dbig = {state, group, total}: state 1 =
// prepared, 2 = lists overflowed (k_decimate rebuilds on its own), 0 = idle.
// ---------------------------------------------------------------------------
constexpr int DEC_BIG_MIN = 4096;

__global__ void __launch_bounds__(1024) k_decbig_setup(EngineView v)
{
    __shared__ int s_w[32];
    __shared__ int s_carry;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    if (tid == 0) { v.dbig[0] = 0; s_carry = 0; }
    if (v.ctr[CTR_NREADY] != 1) return;
    const int g = v.ready[0];
    const GroupDesc gd = v.gr[g];
    __syncthreads();
    // exclusive prefix of the members' chosen counts -> dcpre
    for (int i0 = 0; i0 < gd.n_clouds; i0 += 1024) {
        const int i = i0 + tid;
        const int x = (i < gd.n_clouds) ? v.ns[gd.cloud_begin + i] : 0;
        int incl = x;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(FULL, incl, o);
            if (lane >= o) incl += y;
        }
        if (lane == 31) s_w[warp] = incl;
        __syncthreads();
        int pre = 0, tot = 0;
        for (int w = 0; w < 32; ++w) {
            pre += (w < warp) ? s_w[w] : 0;
            tot += s_w[w];
        }
        const int carry = s_carry;
        if (i < gd.n_clouds) v.dcpre[i] = carry + pre + incl - x;
        __syncthreads();
        if (tid == 0) s_carry = carry + tot;
        __syncthreads();
    }
    const int total = s_carry;
    if (total <= DEC_BIG_MIN) return;
    const int hbits = v.dec_hbits[g];
    int32_t* bstart = v.dbstart + v.dec_hoff[g];
    for (int h = tid; h <= (1 << hbits); h += 1024) bstart[h] = 0;
    if (tid == 0) {
        v.dcpre[gd.n_clouds] = total;
        v.dbig[1] = g;
        v.dbig[2] = total;
        v.dbig[0] = 1;
    }
}

template <int DIM>
__global__ void __launch_bounds__(256) k_decbig_gather(EngineView v)
{
    if (v.dbig[0] != 1) return;
    const int g = v.dbig[1], total = v.dbig[2];
    const GroupDesc gd = v.gr[g];
    const CloudDesc c0 = v.cl[gd.cloud_begin];
    const double inv = 1.0 / (2.0 * (double)c0.r2 * (1.0 + 1.0 / 1024.0));
    const uint32_t hmask = (1u << v.dec_hbits[g]) - 1;
    float* X = v.dx + gd.s_scratch * DIM;
    int32_t* cell = v.dcell + gd.s_scratch * DIM;
    int32_t* bstart = v.dbstart + v.dec_hoff[g];
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < total; t += gridDim.x * blockDim.x) {
        int lo = 0, hi = gd.n_clouds - 1;  // last member with dcpre <= t
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (v.dcpre[mid] <= t) lo = mid;
            else hi = mid - 1;
        }
        const CloudDesc cd = v.cl[gd.cloud_begin + lo];
        const int local = t - v.dcpre[lo];
        int cc[DIM];
#pragma unroll
        for (int d = 0; d < DIM; ++d) {
            const float x = v.S[(cd.s_off + local) * DIM + d];
            X[(int64_t)t * DIM + d] = x;
            cc[d] = cell_of(x, inv);
            cell[(int64_t)t * DIM + d] = cc[d];
        }
        atomicAdd(&bstart[(cell_hash<DIM>(cc) & hmask) + 1], 1);
    }
}

// exclusive prefix over the big group's buckets (bstart[b] -> start of bucket b)
__global__ void __launch_bounds__(1024) k_decbig_scan_buckets(EngineView v)
{
    if (v.dbig[0] != 1) return;
    __shared__ int s_w[32];
    __shared__ int s_carry;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int g = v.dbig[1];
    const int n = (1 << v.dec_hbits[g]) + 1;
    int32_t* bstart = v.dbstart + v.dec_hoff[g];
    if (tid == 0) s_carry = 0;
    __syncthreads();
    for (int i0 = 0; i0 < n; i0 += 1024) {
        const int i = i0 + tid;
        const int x = (i < n) ? bstart[i] : 0;
        int incl = x;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(FULL, incl, o);
            if (lane >= o) incl += y;
        }
        if (lane == 31) s_w[warp] = incl;
        __syncthreads();
        int pre = 0, tot = 0;
        for (int w = 0; w < 32; ++w) {
            pre += (w < warp) ? s_w[w] : 0;
            tot += s_w[w];
        }
        const int carry = s_carry;
        if (i < n) bstart[i] = carry + pre + incl;  // inclusive of the shifted counts
        __syncthreads();
        if (tid == 0) s_carry = carry + tot;
        __syncthreads();
    }
}

template <int DIM>
__global__ void __launch_bounds__(256) k_decbig_fill(EngineView v)
{
    if (v.dbig[0] != 1) return;
    const int g = v.dbig[1], total = v.dbig[2];
    const GroupDesc gd = v.gr[g];
    const uint32_t hmask = (1u << v.dec_hbits[g]) - 1;
    const int32_t* cell = v.dcell + gd.s_scratch * DIM;
    int32_t* items = v.ditems + gd.s_scratch;
    int32_t* bstart = v.dbstart + v.dec_hoff[g];
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < total; t += gridDim.x * blockDim.x) {
        int cc[DIM];
#pragma unroll
        for (int d = 0; d < DIM; ++d) cc[d] = cell[(int64_t)t * DIM + d];
        items[atomicAdd(&bstart[cell_hash<DIM>(cc) & hmask], 1)] = t;
    }
}

template <int DIM>
__global__ void __launch_bounds__(256) k_decbig_count(EngineView v)
{
    if (v.dbig[0] != 1) return;
    const int g = v.dbig[1], total = v.dbig[2];
    const GroupDesc gd = v.gr[g];
    const CloudDesc c0 = v.cl[gd.cloud_begin];
    const float rsq = sqr_rn(c0.r2);
    const float rsq4 = __fmul_rn(4.0f, rsq);
    const uint32_t hmask = (1u << v.dec_hbits[g]) - 1;
    const float* X = v.dx + gd.s_scratch * DIM;
    const int32_t* cell = v.dcell + gd.s_scratch * DIM;
    const int32_t* items = v.ditems + gd.s_scratch;
    const int32_t* bstart = v.dbstart + v.dec_hoff[g];
    int32_t* c1 = v.dc1 + gd.s_scratch;
    int32_t* c2 = v.dc2 + gd.s_scratch;
    int32_t* nb_off = v.dnb_off + gd.s_scratch + g;
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < total; t += gridDim.x * blockDim.x) {
        int n1 = 1, n2 = 1;
        dec_for_neighbours<DIM>(t, X, cell, items, bstart, hmask, rsq, rsq4,
                                [&](int, bool w1) { ++n2; n1 += w1; });
        c1[t] = n1;
        c2[t] = n2;
        nb_off[t] = n2 - 1;
    }
}

// exclusive prefix of the list lengths; flags overflow of the list capacity
__global__ void __launch_bounds__(1024) k_decbig_scan_lists(EngineView v)
{
    if (v.dbig[0] != 1) return;
    __shared__ int s_w[32];
    __shared__ int s_carry;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int g = v.dbig[1], total = v.dbig[2];
    const GroupDesc gd = v.gr[g];
    int32_t* nb_off = v.dnb_off + gd.s_scratch + g;
    if (tid == 0) s_carry = 0;
    __syncthreads();
    for (int i0 = 0; i0 < total; i0 += 1024) {
        const int i = i0 + tid;
        const int x = (i < total) ? nb_off[i] : 0;
        int incl = x;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(FULL, incl, o);
            if (lane >= o) incl += y;
        }
        if (lane == 31) s_w[warp] = incl;
        __syncthreads();
        int pre = 0, tot = 0;
        for (int w = 0; w < 32; ++w) {
            pre += (w < warp) ? s_w[w] : 0;
            tot += s_w[w];
        }
        const int carry = s_carry;
        if (i < total) nb_off[i] = carry + pre + incl - x;
        __syncthreads();
        if (tid == 0) s_carry = carry + tot;
        __syncthreads();
    }
    if (tid == 0) {
        nb_off[total] = s_carry;
        if ((int64_t)s_carry > (int64_t)v.dec_nb_pp * gd.s_cap) v.dbig[0] = 2;
    }
}

template <int DIM>
__global__ void __launch_bounds__(256) k_decbig_lists(EngineView v)
{
    if (v.dbig[0] != 1) return;
    const int g = v.dbig[1], total = v.dbig[2];
    const GroupDesc gd = v.gr[g];
    const CloudDesc c0 = v.cl[gd.cloud_begin];
    const float rsq = sqr_rn(c0.r2);
    const float rsq4 = __fmul_rn(4.0f, rsq);
    const uint32_t hmask = (1u << v.dec_hbits[g]) - 1;
    const float* X = v.dx + gd.s_scratch * DIM;
    const int32_t* cell = v.dcell + gd.s_scratch * DIM;
    const int32_t* items = v.ditems + gd.s_scratch;
    const int32_t* bstart = v.dbstart + v.dec_hoff[g];
    const int32_t* nb_off = v.dnb_off + gd.s_scratch + g;
    int32_t* nb = v.dnb + (int64_t)v.dec_nb_pp * gd.s_scratch;
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < total; t += gridDim.x * blockDim.x) {
        int k = nb_off[t];
        dec_for_neighbours<DIM>(t, X, cell, items, bstart, hmask, rsq, rsq4,
                                [&](int q, bool w1) { nb[k++] = w1 ? (q | (int)0x80000000) : q; });
    }
}

template <int DIM>
cudaError_t launch_decbig(const EngineView& v, cudaStream_t st)
{
    const int grid = v.n_sms * 8;
    k_decbig_setup<<<1, 1024, 0, st>>>(v);
    k_decbig_gather<DIM><<<grid, 256, 0, st>>>(v);
    k_decbig_scan_buckets<<<1, 1024, 0, st>>>(v);
    k_decbig_fill<DIM><<<grid, 256, 0, st>>>(v);
    k_decbig_count<DIM><<<grid, 256, 0, st>>>(v);
    k_decbig_scan_lists<<<1, 1024, 0, st>>>(v);
    k_decbig_lists<DIM><<<grid, 256, 0, st>>>(v);
    return cudaGetLastError();
}

__device__ void loop_condition(const EngineView& v, cudaGraphConditionalHandle h, int use_handle,
                               int count_iter);

// one CTA per group queued by the control step in this iteration; with_cond:
// the last CTA to finish then runs the loop-condition step (the phases and
// chosen counts of every group are final by then)
template <int DIM, int BLOCK>
__global__ void __launch_bounds__(BLOCK) k_decimate(EngineView v, cudaGraphConditionalHandle h,
                                                    int with_cond, int use_handle)
{
    pdl_enter();
    __shared__ int s_last;
    const int nready = v.ctr[CTR_NREADY];
    for (int r = blockIdx.x; r < nready; r += gridDim.x) decimate_group<DIM, BLOCK>(v, v.ready[r]);
    if (!with_cond) return;
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) s_last = atomicAdd(&v.ctr[CTR_DEC_DONE], 1) == (int)gridDim.x - 1;
    __syncthreads();
    if (!s_last) return;
    __threadfence();
    if (threadIdx.x == 0) v.ctr[CTR_DEC_DONE] = 0;
    loop_condition(v, h, use_handle, 1);
}

// ---------------------------------------------------------------------------
// loop condition: any unfinished cloud?  Sets the graph WHILE handle (graph
// mode) and/or leaves the count in ctr[CTR_ACTIVE] for the host (plain mode).
// Run by one whole CTA (any size up to 1024 threads).
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(1024) k_loopcond(EngineView v, cudaGraphConditionalHandle h,
                                                   int use_handle, int count_iter)
{
    loop_condition(v, h, use_handle, count_iter);
}

__device__ void loop_condition(const EngineView& v, cudaGraphConditionalHandle h, int use_handle,
                               int count_iter)
{
    __shared__ int s_act;
    __shared__ int s_w[32][ACT_KINDS + 1];
    __shared__ int s_carry[ACT_KINDS + 1];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    if (tid == 0) {
        s_act = 0;
        for (int q = 0; q <= ACT_KINDS; ++q) s_carry[q] = 0;
    }
    __syncthreads();
    int act = 0;
    for (int c = tid; c < v.n_clouds; c += blockDim.x) act += (v.phase[c] != PH_DONE);
    if (act) atomicAdd(&s_act, act);
    // work lists of the next iteration: evolving clouds, prefixes of their
    // chunks, chosen-point blocks and chosen slots
    const int nc = v.n_clouds;
    for (int c0 = 0; c0 < nc; c0 += blockDim.x) {
        const int c = c0 + tid;
        const bool ev = (c < nc) && v.phase[c] == PH_EVOLVE;
        int x[ACT_KINDS + 1];
        x[0] = ev ? 1 : 0;
        const int rows = ev ? v.cl[c].n_chunks : 0;
        const int nkb = ev ? (v.ns[c] + KBLK - 1) / KBLK : 0;
        x[1 + ACT_CHUNK] = rows;
        x[1 + ACT_KBLK] = rows > SCAN_ROWS_WARP ? nkb : 0;
        x[1 + ACT_KBLK_WARP] = rows > SCAN_ROWS_WARP ? 0 : nkb;
        x[1 + ACT_SLOT] = ev ? v.ns[c] : 0;
        int incl[ACT_KINDS + 1];
#pragma unroll
        for (int q = 0; q <= ACT_KINDS; ++q) {
            incl[q] = x[q];
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const int y = __shfl_up_sync(FULL, incl[q], o);
                if (lane >= o) incl[q] += y;
            }
            if (lane == 31) s_w[warp][q] = incl[q];
        }
        __syncthreads();
        int excl[ACT_KINDS + 1], tot[ACT_KINDS + 1];
#pragma unroll
        for (int q = 0; q <= ACT_KINDS; ++q) {
            int pre = 0, t = 0;
            for (int w = 0; w < (int)(blockDim.x >> 5); ++w) {
                pre += (w < warp) ? s_w[w][q] : 0;
                t += s_w[w][q];
            }
            excl[q] = s_carry[q] + pre + incl[q] - x[q];
            tot[q] = t;
        }
        if (ev) {
            v.act_cloud[excl[0]] = c;
#pragma unroll
            for (int q = 0; q < ACT_KINDS; ++q) v.act_pre[q * (nc + 1) + excl[0]] = excl[1 + q];
        }
        __syncthreads();
        if (tid == 0) {
#pragma unroll
            for (int q = 0; q <= ACT_KINDS; ++q) s_carry[q] += tot[q];
        }
        __syncthreads();
    }
    if (tid == 0) {
        const int nact = s_carry[0];
        for (int q = 0; q < ACT_KINDS; ++q) v.act_pre[q * (nc + 1) + nact] = s_carry[1 + q];
        v.ctr[CTR_NACT] = nact;
        v.ctr[CTR_WORK] = 0;
        v.ctr[CTR_NREADY] = 0;
        v.ctr[CTR_NBIG] = 0;
        v.ctr[CTR_TILE_HEAVY] = 0;
        const int it = v.ctr[CTR_ITERS] + (count_iter ? 1 : 0);
        v.ctr[CTR_ITERS] = it;
        int a = s_act;
        if (it >= v.max_iters && a > 0) {
            v.ctr[CTR_ERR] |= ERRB_EVOLVE_CAP;
            a = 0;
        }
        v.ctr[CTR_ACTIVE] = a;
        if (use_handle) cudaGraphSetConditional(h, a > 0 ? 1u : 0u);
    }
}

// chosen counts are given in v.ns: evolving phase for non-empty clouds, or
// (queue_decimation) converged phase with every group queued for decimation
__global__ void k_set_given(EngineView v, int queue_decimation)
{
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c < v.n_clouds) {
        if (queue_decimation) v.phase[c] = PH_CONVERGED;
        else v.phase[c] = (v.ns[c] > 0) ? PH_EVOLVE : PH_DONE;
    }
    if (queue_decimation && c < v.n_groups) {
        v.ready[c] = c;
        v.group_conv[c] = v.gr[c].n_clouds;
    }
    if (c == 0) v.ctr[CTR_NREADY] = queue_decimation ? v.n_groups : 0;
}

__global__ void k_reset(EngineView v)
{
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c < CTR_COUNT && blockIdx.x == 0) v.ctr[c] = 0;
    if (c == 0) v.dbig[0] = 0;
    if (c < v.n_groups) v.group_conv[c] = 0;
    if (c >= v.n_clouds) return;
    v.kbdone[c] = 0;
    v.cont[c] = 0;
    v.passes[c] = 0;
    v.total_passes[c] = 0;
    v.outer[c] = 0;
    v.err[c] = 0;
    v.pairs[c] = 0;
}

template <int DIM, int BLOCK, int ITEMS>
cudaError_t set_assign_attrs(int dyn)
{
    return cudaFuncSetAttribute(k_assign<DIM, BLOCK, ITEMS>,
                                cudaFuncAttributeMaxDynamicSharedMemorySize, dyn);
}

// persistent grid of k_assign_cull: every resident CTA, at most one per item
template <int DIM, int ITEMS>
cudaError_t launch_assign_cull(const EngineView& v, cudaStream_t st)
{
    static std::atomic<int> per_sm{0};
    int b = per_sm.load(std::memory_order_relaxed);
    if (b == 0) {
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, k_assign_cull<DIM, ITEMS>, AC_BLOCK, 0) !=
                cudaSuccess || b < 1)
            b = 1;
        per_sm.store(b, std::memory_order_relaxed);
    }
    const int subs = (v.chunk_pts + AC_BLOCK * ITEMS - 1) / (AC_BLOCK * ITEMS);
    if (subs & (subs - 1)) return cudaErrorInvalidValue;  // the kernel's block bounds need 2^k
    const int64_t items = (int64_t)v.n_chunks * subs;
    const int g = (int)std::max<int64_t>(1, std::min<int64_t>(items, (int64_t)v.n_sms * b));
    k_assign_cull<DIM, ITEMS><<<g, AC_BLOCK, 0, st>>>(v);
    return cudaGetLastError();
}

template <int DIM>
cudaError_t prepare_pass_dim(const EngineView& v, const TuneParams& tp)
{
    const int hist_bytes = v.hist_smem * 4;
    cudaError_t e = cudaErrorInvalidValue;
#define RD_PREP_CASE(B, I) \
    if (tp.block == B && tp.items == I) e = set_assign_attrs<DIM, B, I>(hist_bytes);
    RD_PREP_CASE(128, 8) RD_PREP_CASE(128, 4) RD_PREP_CASE(256, 4) RD_PREP_CASE(256, 8)
    RD_PREP_CASE(128, 16)
#undef RD_PREP_CASE
    if (e != cudaSuccess) return e;
    e = cudaFuncSetAttribute(k_decimate<DIM, 512>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             dec_smem_bytes(v));
    if (e != cudaSuccess) return e;
    return cudaFuncSetAttribute(k_scatter_cta<DIM>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                scatter_cta_smem_bytes(v));
}

// launch with programmatic stream serialisation (pdl != 0): the kernel may
// start while the previous kernel on the stream drains; it waits in
// pdl_enter(). Single-cloud passes (small, latency-bound grids) gain from it
// (33.7 -> 33.5 ms per 1M-point helix solve); batches of thousands of clouds
// lose 1% with it, so they launch plainly.
template <typename... KArgs, typename... Args>
static cudaError_t launch_pdl(int pdl, void (*kernel)(KArgs...), int grid, int block, size_t smem,
                              cudaStream_t st, Args... args)
{
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(grid);
    cfg.blockDim = dim3(block);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = pdl ? 1 : 0;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, kernel, args...);
}

template <int DIM>
cudaError_t launch_pass_dim(const EngineView& v, const TuneParams& tp, int assign_grid,
                            const LoopCond& lc, cudaStream_t st, cudaEvent_t a0, cudaEvent_t a1)
{
    const int hist_bytes = v.hist_smem * 4;
    const int sms = v.n_sms;
    if (a0) cudaEventRecord(a0, st);
    if (v.cull) {
        cudaError_t e;
        if (tp.cull_items == 2) e = launch_assign_cull<DIM, 2>(v, st);
        else if (tp.cull_items == 8) e = launch_assign_cull<DIM, 8>(v, st);
        else e = launch_assign_cull<DIM, 4>(v, st);
        if (e != cudaSuccess) return e;
    } else {
#define RD_ASSIGN_CASE(B, I)                                                                  \
    if (tp.block == B && tp.items == I) {                                                     \
        k_assign<DIM, B, I><<<assign_grid, B, hist_bytes, st>>>(v);                           \
    } else
    RD_ASSIGN_CASE(128, 8)
    RD_ASSIGN_CASE(128, 4)
    RD_ASSIGN_CASE(256, 4)
    RD_ASSIGN_CASE(256, 8)
    RD_ASSIGN_CASE(128, 16)
    { return cudaErrorInvalidValue; }
#undef RD_ASSIGN_CASE
    }
    if (a1) cudaEventRecord(a1, st);
    // fixed grids; every kernel walks only the current work lists
    // every kernel after the assignment is a programmatic dependent of the one
    // before it (pdl_enter) when a single cloud evolves
    const int pdl = v.n_clouds == 1;
    cudaError_t e = cudaSuccess;
    if (v.n_kblk > 0)
        e = launch_pdl(pdl, k_chunkscan_cta, std::min(v.n_kblk, sms * 4), CS_W * 32, 0, st, v);
    if (e == cudaSuccess && v.n_kblk_warp > 0)
        e = launch_pdl(pdl, k_chunkscan_warp, std::min((v.n_kblk_warp + CSW_W - 1) / CSW_W, sms * 8),
                       CSW_W * 32, 0, st, v);
    if (e == cudaSuccess && v.n_chunks > 0)
        e = launch_pdl(pdl, k_scatter_cta<DIM>, std::min(v.n_chunks, sms * 8), SCAT_W * 32,
                       scatter_cta_smem_bytes(v), st, v);
    if (e != cudaSuccess) return e;
    if (v.n_slots > 0) {
        // at most (points / SUM_BIG_MIN) keys can be big
        const int big_ctas = (int)std::min<int64_t>(
            ((int64_t)v.n_chunks * v.chunk_pts + SUM_BIG_MIN - 1) / SUM_BIG_MIN, sms);
        e = launch_pdl(pdl, k_sum_shift<DIM>, big_ctas + std::min((v.n_slots + 7) / 8, sms * 8), 256, 0,
                       st, v, big_ctas, 1);
    } else {
        e = launch_pdl(pdl, k_control, std::min((v.n_clouds + 255) / 256, sms), 256, 0, st, v);
    }
    if (e != cudaSuccess) return e;
    return launch_pdl(pdl, k_decimate<DIM, 512>, std::min(v.n_groups, sms * 2), 512, dec_smem_bytes(v),
                      st, v, lc.h, 1, lc.use_handle);
}

template <int DIM>
cudaError_t launch_choose_dim(const EngineView& v, cudaStream_t st)
{
    using CS = ChooseSmem<DIM>;
    constexpr int B = 1024;
    const int bytes = CS::HB * 4 + CS::SCAP * 4 + CS::SCAP * DIM * 4 + B * DIM * 8;
    cudaError_t e =
        cudaFuncSetAttribute(k_choose<DIM, B>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
    if (e != cudaSuccess) return e;
    k_choose<DIM, B><<<v.n_clouds, B, bytes, st>>>(v);
    return cudaGetLastError();
}

// rounds over [0, n): 4096 points first, doubling; needs v.hash (HB ints) and
// surv (n bytes)
template <int DIM>
cudaError_t launch_choose_rounds_dim(const EngineView& v, int c, int n, uint8_t* surv,
                                     int32_t* sel, void* tmp, size_t tmp_bytes, cudaStream_t st)
{
    using CS = ChooseSmem<DIM>;
    constexpr int B = 1024;
    const int bytes = CS::HB * 4 + CS::SCAP * 4 + CS::SCAP * DIM * 4 + B * DIM * 8;
    cudaError_t e = cudaFuncSetAttribute(k_choose_resolve<DIM, B>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
    if (e != cudaSuccess) return e;
    int a = 0, size = 4096, first = 1;
    int32_t* nsel = sel + n;
    while (a < n) {
        const int b = (int)std::min<int64_t>((int64_t)n, (int64_t)a + size);
        if (first) {
            k_choose_resolve<DIM, B><<<1, B, bytes, st>>>(v, c, a, b, nullptr, nullptr, first);
        } else {
            const int grid = std::max(1, std::min((b - a + 255) / 256, 148 * 16));
            k_choose_filter<DIM><<<grid, 256, 0, st>>>(v, c, a, b, surv);
            size_t tb = tmp_bytes;
            e = cub::DeviceSelect::Flagged(tmp, tb, cub::CountingInputIterator<int32_t>(a), surv, sel,
                                           nsel, b - a, st);
            if (e != cudaSuccess) return e;
            k_choose_resolve<DIM, B><<<1, B, bytes, st>>>(v, c, a, b, sel, nsel, first);
        }
        a = b;
        size = (int)std::min<int64_t>((int64_t)size * 2, 1 << 30);
        first = 0;
    }
    return cudaGetLastError();
}

}  // namespace

cudaError_t launch_choose_rounds(int dim, const EngineView& v, int c, int n, uint8_t* surv,
                                 int32_t* sel, void* tmp, size_t tmp_bytes, cudaStream_t st)
{
    return with_dim(dim, [&](auto D) {
        return launch_choose_rounds_dim<decltype(D)::value>(v, c, n, surv, sel, tmp, tmp_bytes, st);
    });
}

int choose_hash_buckets() { return ChooseSmem<2>::HB; }

size_t choose_select_scratch_bytes(int64_t n)
{
    size_t tb = 0;
    cub::DeviceSelect::Flagged(nullptr, tb, cub::CountingInputIterator<int32_t>(0), (const uint8_t*)nullptr,
                               (int32_t*)nullptr, (int32_t*)nullptr, (int)std::max<int64_t>(n, 1));
    return tb + 256;
}

cudaError_t launch_choose(int dim, const EngineView& v, cudaStream_t st)
{
    return with_dim(dim, [&](auto D) { return launch_choose_dim<decltype(D)::value>(v, st); });
}

cudaError_t prepare_pass(int dim, const EngineView& v, const TuneParams& tp)
{
    return with_dim(dim, [&](auto D) { return prepare_pass_dim<decltype(D)::value>(v, tp); });
}

cudaError_t launch_pass(int dim, const EngineView& v, const TuneParams& tp, int assign_grid,
                        const LoopCond& lc, cudaStream_t st, cudaEvent_t a0, cudaEvent_t a1)
{
    return with_dim(dim, [&](auto D) {
        return launch_pass_dim<decltype(D)::value>(v, tp, assign_grid, lc, st, a0, a1);
    });
}

cudaError_t launch_loopcond(const EngineView& v, cudaGraphConditionalHandle h, int use_handle,
                            cudaStream_t st, int count_iter)
{
    k_loopcond<<<1, 1024, 0, st>>>(v, h, use_handle, count_iter);
    return cudaGetLastError();
}

static std::atomic<int> g_tile_cl_on{1}, g_tile_cl_min{TCL_MIN_POINTS}, g_tile_seg_min{TSEG_MIN};
TileClusterParams tile_cluster_defaults() { return TileClusterParams{true, TCL_MIN_POINTS, TSEG_MIN}; }
TileClusterParams tile_cluster_params()
{
    return TileClusterParams{g_tile_cl_on.load() != 0, g_tile_cl_min.load(), g_tile_seg_min.load()};
}
void set_tile_cluster_params(const TileClusterParams& p)
{
    g_tile_cl_on.store(p.enabled ? 1 : 0);
    g_tile_cl_min.store(p.min_points);
    g_tile_seg_min.store(p.seg_min);
}

// launch configuration of the cluster tile kernel: one CTA per resident slot
// (TCL-CTA clusters), dynamic shared memory as tile_cluster_smem_bytes
template <int DIM>
static void tile_cl_config(cudaLaunchConfig_t& cfg, cudaLaunchAttribute* at, int grid)
{
    std::memset(&cfg, 0, sizeof(cfg));
    cfg.gridDim = dim3(grid, 1, 1);
    cfg.blockDim = dim3(256, 1, 1);
    cfg.dynamicSmemBytes = tile_cluster_smem_bytes(DIM);
    at[0].id = cudaLaunchAttributeClusterDimension;
    at[0].val.clusterDim.x = TCL;
    at[0].val.clusterDim.y = 1;
    at[0].val.clusterDim.z = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
}

template <int DIM>
static cudaError_t tile_cl_prepare(int* cl_grid)
{
    cudaError_t e = cudaFuncSetAttribute(k_tile_evolve_cl<DIM, 256>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         tile_cluster_smem_bytes(DIM));
    if (e != cudaSuccess) return e;
    cudaLaunchConfig_t cfg;
    cudaLaunchAttribute at[1];
    tile_cl_config<DIM>(cfg, at, TCL);
    int ncl = 0;
    e = cudaOccupancyMaxActiveClusters(&ncl, k_tile_evolve_cl<DIM, 256>, &cfg);
    if (e != cudaSuccess) return e;
    *cl_grid = (ncl > 0) ? ncl * TCL : 0;
    return cudaSuccess;
}

cudaError_t prepare_tile_pass(int dim, const EngineView& v, int* cl_grid)
{
    *cl_grid = 0;
    return with_dim(dim, [&](auto D) {
        constexpr int DIM = decltype(D)::value;
        cudaError_t e = cudaFuncSetAttribute(k_tile_evolve<DIM, 256>,
                                             cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             tile_evolve_smem_bytes(DIM));
        if (e != cudaSuccess) return e;
        if (v.n_heavy > 0) {
            e = tile_cl_prepare<DIM>(cl_grid);
            if (e != cudaSuccess) return e;
        }
        return cudaFuncSetAttribute(k_decimate<DIM, 512>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    dec_smem_bytes(v));
    });
}

cudaError_t launch_tile_pass(int dim, const EngineView& v, const LoopCond& lc, cudaStream_t st,
                             cudaEvent_t a0, cudaEvent_t a1)
{
    const int smem = tile_evolve_smem_bytes(dim);
    const int grid = std::max(1, std::min(v.n_clouds, v.n_sms * 3));
    const int dgrid = std::max(1, std::min(v.n_groups, v.n_sms * 2));
    return with_dim(dim, [&](auto D) {
        constexpr int DIM = decltype(D)::value;
        if (a0) cudaEventRecord(a0, st);
        if (v.tile_cl_grid > 0) {
            cudaLaunchConfig_t cfg;
            cudaLaunchAttribute at[1];
            tile_cl_config<DIM>(cfg, at, v.tile_cl_grid);
            cfg.stream = st;
            const cudaError_t e = cudaLaunchKernelEx(&cfg, k_tile_evolve_cl<DIM, 256>, v);
            if (e != cudaSuccess) return e;
        } else {
            k_tile_evolve<DIM, 256><<<grid, 256, smem, st>>>(v);
        }
        if (a1) cudaEventRecord(a1, st);
        launch_decbig<DIM>(v, st);
        k_decimate<DIM, 512><<<dgrid, 512, dec_smem_bytes(v), st>>>(v, lc.h, 1, lc.use_handle);
        return cudaGetLastError();
    });
}

template <int DIM>
__global__ void __launch_bounds__(32) k_ordered_sum(const float* P, const int32_t* idx, int n,
                                                   float* out, int method)
{
    __shared__ float s_buf[SUM_BP * DIM];
    __shared__ int s_idx[SUM_BP];
    const int lane = threadIdx.x;
    const float r = (method == 1) ? fold_members_par<DIM>(idx, n, P, lane)
                                  : fold_members<DIM>(idx, n, P, s_buf, s_idx, lane);
    if (lane < DIM) out[lane] = r;
}

template <int DIM>
__global__ void __launch_bounds__(256) k_ordered_sum_cta(const float* P, const int32_t* idx, int n,
                                                         float* out)
{
    __shared__ FoldCtaSmem<8, DIM> sm;
    fold_members_cta<8, DIM>(idx, n, P, sm);
    if (threadIdx.x < DIM) out[threadIdx.x] = sm.s[threadIdx.x];
}

template <int DIM, int BLOCK>
__global__ void __launch_bounds__(BLOCK) k_ordered_sum_seg(const float* P, const int32_t* idx, int n,
                                                           float* out)
{
    __shared__ SegFoldSmem<BLOCK / 32, DIM> sm;
    fold_members_seg<BLOCK / 32, DIM>(idx, n, P, sm);
    if (threadIdx.x < DIM) out[threadIdx.x] = sm.out[threadIdx.x];
}

cudaError_t launch_ordered_sum(int dim, const float* P, const int32_t* idx, int n, float* out,
                               int method, cudaStream_t st)
{
    return with_dim(dim, [&](auto D) {
        constexpr int DIM = decltype(D)::value;
        if (method == 3) k_ordered_sum_seg<DIM, 256><<<1, 256, 0, st>>>(P, idx, n, out);
        else if (method == 4) k_ordered_sum_seg<DIM, 1024><<<1, 1024, 0, st>>>(P, idx, n, out);
        else if (method == 2) k_ordered_sum_cta<DIM><<<1, 256, 0, st>>>(P, idx, n, out);
        else k_ordered_sum<DIM><<<1, 32, 0, st>>>(P, idx, n, out, method);
        return cudaGetLastError();
    });
}

cudaError_t launch_set_given(const EngineView& v, int queue_decimation, cudaStream_t st)
{
    const int n = v.n_clouds > v.n_groups ? v.n_clouds : v.n_groups;
    k_set_given<<<(n + 255) / 256, 256, 0, st>>>(v, queue_decimation);
    return cudaGetLastError();
}

cudaError_t launch_decimate(int dim, const EngineView& v, cudaStream_t st)
{
    const int grid = std::max(1, std::min(v.n_groups, v.n_sms * 2));
    const int smem = dec_smem_bytes(v);
    cudaError_t e = cudaSuccess;
    e = with_dim(dim, [&](auto D) {
        constexpr int DIM = decltype(D)::value;
        cudaError_t r = cudaFuncSetAttribute(k_decimate<DIM, 512>,
                                             cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
        if (r == cudaSuccess) k_decimate<DIM, 512><<<grid, 512, smem, st>>>(v, 0, 0, 0);
        return r;
    });
    if (e != cudaSuccess) return e;
    return cudaGetLastError();
}

template <int DIM>
cudaError_t launch_evolve_step_dim(const EngineView& v, const TuneParams& tp, int assign_grid,
                                   cudaStream_t st)
{
    const int hist_bytes = v.hist_smem * 4;
    const int sms = v.n_sms;
#define RD_ASSIGN_CASE(B, I) \
    if (tp.block == B && tp.items == I) k_assign<DIM, B, I><<<assign_grid, B, hist_bytes, st>>>(v); else
    RD_ASSIGN_CASE(128, 8) RD_ASSIGN_CASE(128, 4) RD_ASSIGN_CASE(256, 4) RD_ASSIGN_CASE(256, 8)
    RD_ASSIGN_CASE(128, 16)
    { return cudaErrorInvalidValue; }
#undef RD_ASSIGN_CASE
    if (v.n_kblk > 0) k_chunkscan_cta<<<std::min(v.n_kblk, sms * 4), CS_W * 32, 0, st>>>(v);
    if (v.n_kblk_warp > 0)
        k_chunkscan_warp<<<std::min((v.n_kblk_warp + CSW_W - 1) / CSW_W, sms * 8), CSW_W * 32, 0, st>>>(v);
    if (v.n_chunks > 0)
        k_scatter_cta<DIM><<<std::min(v.n_chunks, sms * 8), SCAT_W * 32, scatter_cta_smem_bytes(v), st>>>(v);
    if (v.n_slots > 0) {
        // at most (points / SUM_BIG_MIN) keys can be big
        const int big_ctas = (int)std::min<int64_t>(
            ((int64_t)v.n_chunks * v.chunk_pts + SUM_BIG_MIN - 1) / SUM_BIG_MIN, sms);
        k_sum_shift<DIM><<<big_ctas + std::min((v.n_slots + 7) / 8, sms * 8), 256, 0, st>>>(v, big_ctas, 0);
    }
    return cudaGetLastError();
}

cudaError_t launch_evolve_step(int dim, const EngineView& v, const TuneParams& tp, int assign_grid,
                               cudaStream_t st)
{
    return with_dim(dim, [&](auto D) {
        return launch_evolve_step_dim<decltype(D)::value>(v, tp, assign_grid, st);
    });
}

cudaError_t launch_reset(const EngineView& v, cudaStream_t st)
{
    int n = v.n_clouds > CTR_COUNT ? v.n_clouds : CTR_COUNT;
    n = n > v.n_groups ? n : v.n_groups;
    k_reset<<<(n + 255) / 256, 256, 0, st>>>(v);
    return cudaGetLastError();
}

bool tune_supported(int dim, const TuneParams& tp)
{
    (void)dim;
    const bool cull_ok = tp.cull_items == 2 || tp.cull_items == 4 || tp.cull_items == 8;
    return cull_ok && ((tp.block == 128 && (tp.items == 4 || tp.items == 8 || tp.items == 16)) ||
                       (tp.block == 256 && (tp.items == 4 || tp.items == 8)));
}

int assign_smem_bytes(int dim, const TuneParams& tp, int hist_ints)
{
    (void)tp;
    const int dp = (dim == 3) ? 4 : dim;
    return ASSIGN_TS * dp * 4 + 16 + hist_ints * 4;
}

template <int DIM, int B, int I>
static int occ_of(int dyn)
{
    int nb = 0;
    if (set_assign_attrs<DIM, B, I>(dyn) != cudaSuccess) return 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_assign<DIM, B, I>, B, dyn);
    return nb;
}

int max_assign_blocks_per_sm(int dim, const TuneParams& tp, int hist_ints)
{
    const int dyn = hist_ints * 4;
#define RD_OCC(D, B, I) \
    if (dim == D && tp.block == B && tp.items == I) return occ_of<D, B, I>(dyn);
    RD_OCC(1, 128, 8) RD_OCC(1, 128, 4) RD_OCC(1, 256, 4) RD_OCC(1, 256, 8) RD_OCC(1, 128, 16)
    RD_OCC(2, 128, 8) RD_OCC(2, 128, 4) RD_OCC(2, 256, 4) RD_OCC(2, 256, 8) RD_OCC(2, 128, 16)
    RD_OCC(3, 128, 8) RD_OCC(3, 128, 4) RD_OCC(3, 256, 4) RD_OCC(3, 256, 8) RD_OCC(3, 128, 16)
    RD_OCC(4, 128, 8) RD_OCC(4, 128, 4) RD_OCC(4, 256, 4) RD_OCC(4, 256, 8) RD_OCC(4, 128, 16)
#undef RD_OCC
    return 0;
}

}  // namespace rdb
