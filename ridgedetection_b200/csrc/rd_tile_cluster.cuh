// rd_tile_cluster.cuh -- cluster-cooperative evolve of the heavy tiles of a
// tiled run (included by rd_kernels.cu after the one-CTA tile kernel).
//
// A tiled run evolves every leaf tile over its own points plus its r1 halo
// (rd/cpu/brute_force/evolve.hpp:345-399 over tile.hpp:167-176).  On a dense
// cloud a few tiles hold hundreds of thousands of evolve points (the halo box
// is several times the tile's area when r1 is close to the tile edge), and one
// CTA evolving such a tile through all its passes is the critical path of the
// whole launch.  Here a thread-block cluster of TCL CTAs evolves one heavy
// tile, pass by pass, with the same results bit for bit:
//
//   assignment   CTA r takes the r-th TCL-th of the tile's points (index
//                order), its warps sub-ranges of that; per-warp key counts;
//   grouping     per-CTA key counts are exchanged through distributed shared
//                memory; every CTA derives the key bases and the offset of its
//                own members inside each key, so the stable placement into
//                Pg (index order inside every key) needs no further exchange;
//   folds        a key with tile_seg_min+ members is folded in TCL x W
//                segments of its member list, one per warp of the cluster: each
//                warp folds its segment from a speculative start (the FP64 sum
//                of the members before it) and records a trace, and one warp
//                replays the traces in order from the exact start
//                (rd_segfold.cuh).  Smaller keys are folded whole by the CTA
//                that owns them (warp fold, or the CTA's segmented fold);
//   shift        the owner of each key applies the movement test; the new
//                coordinates and moved flags are gathered by every CTA, so all
//                CTAs take the same loop decision.
//
// Light tiles are evolved by single CTAs of the same launch (tile_evolve_one)
// once the heavy tiles are handed out.  Every branch that precedes a cluster
// barrier depends only on values that are identical in all CTAs of the
// cluster, so every CTA reaches every barrier.
#pragma once

#include <cooperative_groups.h>

namespace rdb {
namespace {

namespace cg = cooperative_groups;

constexpr int TCL = 8;                  // CTAs per cluster (portable size)
constexpr int TCL_MIN_POINTS = 100000;  // default: evolve points of a tile evolved by a cluster
constexpr int TSEG_MIN = 8192;          // default: members of a key folded across the cluster
constexpr int TSEG_KEYS = 4;            // such keys per pass (the first in key order)
constexpr int TCL_W = 8;                // warps per CTA of the cluster kernel (256 threads)

template <int DIM>
struct ClusterSmem {
    int ccnt[TILE_NS_MAX + 1];       // this CTA's members per key (read by the cluster)
    int kbefore[TILE_NS_MAX + 1];    // members of key k placed by lower-ranked CTAs
    int kcnt[TILE_NS_MAX + 1];       // members per key in the tile
    float res[TILE_NS_MAX][DIM];     // new coordinates of the keys this CTA folds
    int res_moved[TILE_NS_MAX];
    int segk[TSEG_KEYS];             // keys folded across the cluster in this pass
    double part[TSEG_KEYS][TCL_W][DIM];  // FP64 sums of this CTA's warp segments
    double seg64[TSEG_KEYS][DIM];    // and their total
    SegTrace wtr[TSEG_KEYS][TCL_W][DIM];
    int segmv[TSEG_KEYS][DIM];       // a segmented key's coordinate moved
    int nseg;
    int tile;
};

// dynamic shared memory of the cluster kernel: the one-CTA layout, then
// ClusterSmem
constexpr int tile_cluster_base(int dim) { return (tile_evolve_smem_bytes(dim) + 255) / 256 * 256; }

inline int tile_cluster_smem_bytes(int dim)
{
    const int base = tile_cluster_base(dim);
    const int cs[RD_MAX_DIM + 1] = {0, (int)sizeof(ClusterSmem<1>), (int)sizeof(ClusterSmem<2>),
                                    (int)sizeof(ClusterSmem<3>), (int)sizeof(ClusterSmem<4>)};
    return base + cs[dim_supported(dim) ? dim : 2];
}

// The cluster evolves heavy tile c to convergence (see the file comment).
template <int DIM, int BLOCK>
__device__ void tile_evolve_cluster(const EngineView& v, const int c, unsigned char* dyn,
                                    TileCtaSmem<DIM, BLOCK>& ts, ClusterSmem<DIM>& cs,
                                    cg::cluster_group& cl, const int rank)
{
    constexpr int W = BLOCK / 32;
    constexpr int DP = PadDim<DIM>::v;
    constexpr int KB = 8;
    constexpr float FAR = 1e30f;
    float* sS = reinterpret_cast<float*>(dyn);
    int* hist = reinterpret_cast<int*>(sS + TILE_NS_MAX * DP);
    int* kbase = hist + W * (TILE_NS_MAX + 1);
    auto& s_buf = ts.buf;
    auto& s_seg = ts.seg;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    static_assert(W == TCL_W, "the cluster smem holds TCL_W warp segments per CTA");
    const CloudDesc cd = v.cl[c];
    const int n = cd.n_all;
    const int ns = v.ns[c];
    const float* P = v.P + cd.p_off * DIM;
    float* gS = v.S + cd.s_off * DIM;
    int32_t* keys = v.keys + cd.p_off;
    float* Pg = v.Pg + cd.p_off * DP;   // coordinates grouped by key, shared by the cluster
    const float rsq = sqr_rn(cd.r1);
    const int nsp = (ns + KB - 1) / KB * KB;
    __syncthreads();
    for (int e = tid; e < nsp; e += BLOCK)
#pragma unroll
        for (int d = 0; d < DIM; ++d) sS[e * DP + d] = (e < ns) ? gS[(int64_t)e * DIM + d] : FAR;
    const int lo_c = (int)(((int64_t)rank * n) / TCL), hi_c = (int)(((int64_t)(rank + 1) * n) / TCL);
    const int r0 = lo_c + (int)(((int64_t)warp * (hi_c - lo_c)) / W);
    const int r1w = lo_c + (int)(((int64_t)(warp + 1) * (hi_c - lo_c)) / W);
    int pass = 0;
    for (;;) {
        // 1. assignment of this CTA's range (exactly as tile_evolve_one)
        for (int k = lane; k <= ns; k += 32) hist[warp * (TILE_NS_MAX + 1) + k] = 0;
        __syncthreads();
        tile_assign_range<DIM>(P, r0, r1w, sS, ns, nsp, rsq, keys, hist + warp * (TILE_NS_MAX + 1),
                               lane);
        __syncthreads();
        // 2. this CTA's members per key; per-warp offsets inside the CTA
        for (int k = tid; k < ns; k += BLOCK) {
            int run = 0;
            for (int w = 0; w < W; ++w) {
                const int x = hist[w * (TILE_NS_MAX + 1) + k];
                hist[w * (TILE_NS_MAX + 1) + k] = run;
                run += x;
            }
            cs.ccnt[k] = run;
        }
        cl.sync();   // per-CTA counts visible in the cluster
        for (int k = tid; k < ns; k += BLOCK) {
            int tot = 0, before = 0;
            for (int q = 0; q < TCL; ++q) {
                const int x = cl.map_shared_rank(cs.ccnt, q)[k];
                tot += x;
                before += (q < rank) ? x : 0;
            }
            cs.kcnt[k] = tot;
            cs.kbefore[k] = before;
        }
        __syncthreads();
        if (warp == 0) {  // exclusive scan of the tile's counts -> key bases
            int carry = 0;
            for (int k0 = 0; k0 < ns; k0 += 32) {
                const int k = k0 + lane;
                const int x = (k < ns) ? cs.kcnt[k] : 0;
                int incl = x;
#pragma unroll
                for (int o = 1; o < 32; o <<= 1) {
                    const int y = __shfl_up_sync(FULL, incl, o);
                    if (lane >= o) incl += y;
                }
                if (k < ns) kbase[k] = carry + incl - x;
                carry += __shfl_sync(FULL, incl, 31);
            }
            if (lane == 0) kbase[ns] = carry;
            // keys folded across the cluster: the first TSEG_KEYS with
            // tile_seg_min+ members
            int nseg = 0;
            for (int k0 = 0; k0 < ns && nseg < TSEG_KEYS; k0 += 32) {
                const int k = k0 + lane;
                const bool big = (k < ns) && cs.kcnt[k] >= v.tile_seg_min;
                const unsigned bm = __ballot_sync(FULL, big);
                const int pos = nseg + __popc(bm & lanemask_lt());
                if (big && pos < TSEG_KEYS) cs.segk[pos] = k;
                nseg += __popc(bm);
            }
            if (lane == 0) cs.nseg = min(nseg, TSEG_KEYS);
        }
        __syncthreads();
        for (int k = tid; k < ns; k += BLOCK) {
            const int add = kbase[k] + cs.kbefore[k];
            for (int w = 0; w < W; ++w) hist[w * (TILE_NS_MAX + 1) + k] += add;
        }
        __syncthreads();
        // 3. stable placement of this CTA's members (as tile_evolve_one)
        tile_place_range<DIM>(P, keys, r0, r1w, hist + warp * (TILE_NS_MAX + 1), ns, Pg, lane);
        const int nseg = cs.nseg;
        cl.sync();   // Pg complete in the cluster
        // FP64 sums of this CTA's warp segments of every segmented key; a key's
        // list is cut into TCL x W segments, segment g = rank * W + warp
        constexpr int NSEG = TCL * W;
        for (int j = 0; j < nseg; ++j) {
            const int k = cs.segk[j], cnt = cs.kcnt[k];
            const int g = rank * W + warp;
            const int b = (int)(((int64_t)g * cnt) / NSEG), e = (int)(((int64_t)(g + 1) * cnt) / NSEG);
            double acc[DIM];
            warp_sum64_src<DIM>(RowSrc<DIM>{Pg + (int64_t)kbase[k] * DP}, b, e, acc, lane);
            if (lane == 0)
#pragma unroll
                for (int d = 0; d < DIM; ++d) cs.part[j][warp][d] = acc[d];
        }
        __syncthreads();
        if (tid < nseg * DIM) {
            const int j = tid / DIM, d = tid % DIM;
            double t = 0.0;
            for (int w = 0; w < W; ++w) t += cs.part[j][w][d];
            cs.seg64[j][d] = t;
        }
        cl.sync();   // segment sums visible
        // 4a. every warp folds its segment of every segmented key from the
        //     FP64 estimate of the segment's start (segment 0 starts at 0)
        for (int j = 0; j < nseg; ++j) {
            const int k = cs.segk[j], cnt = cs.kcnt[k];
            const int g = rank * W + warp;
            const int b = (int)(((int64_t)g * cnt) / NSEG), e = (int)(((int64_t)(g + 1) * cnt) / NSEG);
            float s0[DIM];
#pragma unroll
            for (int d = 0; d < DIM; ++d) {
                double est = 0.0;
                for (int q = 0; q < rank; ++q) est += cl.map_shared_rank(&cs.seg64[j][0], q)[d];
                for (int w = 0; w < warp; ++w) est += cs.part[j][w][d];
                s0[d] = (g == 0) ? 0.0f : (float)est;
            }
            warp_fold_traced_src<DIM>(RowSrc<DIM>{Pg + (int64_t)kbase[k] * DP}, b, e, s0, cs.wtr[j][warp],
                                      lane);
        }
        // 4b. the other keys this CTA owns (key k belongs to CTA k % TCL)
        auto is_seg = [&](int k) {
            bool r = false;
            for (int j = 0; j < nseg; ++j) r = r || (cs.segk[j] == k);
            return r;
        };
        for (int k = rank; k < ns; k += TCL) {
            const int cnt = cs.kcnt[k];
            if (cnt < FOLD_CTA_MIN || is_seg(k)) continue;
            fold_members_seg_src<W, DIM>(RowSrc<DIM>{Pg + (int64_t)kbase[k] * DP}, cnt, s_seg);
            if (warp == 0) {
                int mv = 0;
                if (lane < DIM) {
                    float cval = sS[k * DP + lane];
                    mv = shift_coord(s_seg.out[lane], cnt, cval);
                    cs.res[k][lane] = cval;
                }
                mv = __any_sync(FULL, mv);
                if (lane == 0) cs.res_moved[k] = mv;
            }
            __syncthreads();
        }
        for (int q = warp; rank + q * TCL < ns; q += W) {
            const int k = rank + q * TCL;
            const int cnt = cs.kcnt[k];
            if (cnt == 0 || cnt >= FOLD_CTA_MIN || is_seg(k)) continue;
            const float sum = fold_rows<DIM, SUM_BP>(Pg + (int64_t)kbase[k] * DP, cnt, s_buf[warp], lane);
            int moved = 0;
            float cval = 0.0f;
            if (lane < DIM) {
                cval = sS[k * DP + lane];
                moved = shift_coord(sum, cnt, cval);
                cs.res[k][lane] = cval;
            }
            moved = __any_sync(FULL, moved);
            if (lane == 0) cs.res_moved[k] = moved;
        }
        cl.sync();   // traces and owned results visible
        // 4c. composition of the segmented keys: key j by CTA j % TCL, warp d,
        //     replaying the TCL x W segment traces in order from the exact start
        //     The warp first copies the NSEG traces of its coordinate from the
        //     cluster's shared memory into this CTA's histogram area (free
        //     until the next pass), so the sequential replay reads local
        //     shared memory instead of making one remote round trip per
        //     segment; coordinates whose traces do not fit there read them
        //     in place.
        constexpr int TR16 = (int)(sizeof(SegTrace) / 16);   // 16-byte words per trace
        constexpr bool STAGE = DIM * NSEG * (int)sizeof(SegTrace) <= W * (TILE_NS_MAX + 1) * 4;
        for (int j = rank; j < nseg; j += TCL) {
            if (warp >= DIM) break;
            const int d = warp;
            const int k = cs.segk[j], cnt = cs.kcnt[k];
            const RowSrc<DIM> rows{Pg + (int64_t)kbase[k] * DP};
            SegTrace* loc = reinterpret_cast<SegTrace*>(hist) + d * NSEG;
            if constexpr (STAGE) {
                for (int t = lane; t < NSEG * TR16; t += 32) {
                    const int g = t / TR16, o = t - (t / TR16) * TR16;
                    const int4* src = reinterpret_cast<const int4*>(
                        &cl.map_shared_rank(&cs, g / W)->wtr[j][g % W][d]);
                    reinterpret_cast<int4*>(loc + g)[o] = src[o];
                }
                __syncwarp();
            }
            auto trace = [&](int g) -> const SegTrace& {
                if constexpr (STAGE) return loc[g];
                else return cl.map_shared_rank(&cs, g / W)->wtr[j][g % W][d];
            };
            float x = trace(0).fin;   // segment 0 started at 0
            for (int g = 1; g < NSEG; ++g) {
                const int b = (int)(((int64_t)g * cnt) / NSEG), e = (int)(((int64_t)(g + 1) * cnt) / NSEG);
                x = replay_segment_src<DIM>(trace(g), rows, b, e, d, x, lane);
            }
            if (lane == 0) {
                float cval = sS[k * DP + d];
                cs.segmv[j][d] = shift_coord(x, cnt, cval);
                cs.res[k][d] = cval;
            }
        }
        cl.sync();   // every key's new coordinates visible
        // 5. gather every key's result from its owner; the same in every CTA
        int moved = 0;
        for (int k = tid; k < ns; k += BLOCK) {
            if (cs.kcnt[k] == 0) continue;
            int jseg = -1;
            for (int j = 0; j < nseg; ++j) jseg = (cs.segk[j] == k) ? j : jseg;
            const ClusterSmem<DIM>* R = cl.map_shared_rank(&cs, jseg >= 0 ? jseg % TCL : k % TCL);
#pragma unroll
            for (int d = 0; d < DIM; ++d) {
                sS[k * DP + d] = R->res[k][d];
                if (jseg >= 0) moved |= R->segmv[jseg][d];
            }
            if (jseg < 0) moved |= R->res_moved[k];
        }
        moved = __syncthreads_or(moved);
        ++pass;
        if (rank == 0 && tid == 0) v.pairs[c] += (unsigned long long)n * (unsigned long long)ns;
        if (!moved) break;
        if (pass >= v.max_passes) {
            if (rank == 0 && tid == 0) v.err[c] |= ERRB_EVOLVE_CAP;
            break;
        }
    }
    if (rank == 0) {
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
    cl.sync();   // no CTA reads this tile's shared state any more
}

// Heavy tiles (tile_order[0..n_heavy), largest first) by whole clusters,
// then the light tiles (tile_order[n_heavy..n_clouds)) by single CTAs.
template <int DIM, int BLOCK>
__global__ void __launch_bounds__(BLOCK) k_tile_evolve_cl(EngineView v)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ TileCtaSmem<DIM, BLOCK> ts;
    __shared__ int s_t;
    ClusterSmem<DIM>& cs = *reinterpret_cast<ClusterSmem<DIM>*>(smem_raw + tile_cluster_base(DIM));
    cg::cluster_group cl = cg::this_cluster();
    const int rank = (int)cl.block_rank();
    const int tid = threadIdx.x;
    for (;;) {
        if (rank == 0 && tid == 0) {
            const int t = atomicAdd(&v.ctr[CTR_TILE_HEAVY], 1);
            int c = (t < v.n_heavy) ? v.tile_order[t] : -1;
            if (c >= 0 && v.phase[c] != PH_EVOLVE) c = -2;   // nothing to evolve: skip
            cs.tile = c;
        }
        cl.sync();
        const int c = *cl.map_shared_rank(&cs.tile, 0);
        cl.sync();   // rank 0 may overwrite its slot from here on
        if (c == -1) break;
        if (c >= 0) tile_evolve_cluster<DIM, BLOCK>(v, c, smem_raw, ts, cs, cl, rank);
    }
    const int n_light = v.n_clouds - v.n_heavy;
    for (;;) {
        if (tid == 0) {
            const int t = atomicAdd(&v.ctr[CTR_WORK], 1);
            s_t = (t < n_light) ? v.tile_order[v.n_heavy + t] : -1;
        }
        __syncthreads();
        const int c = s_t;
        __syncthreads();
        if (c < 0) break;
        if (v.phase[c] == PH_EVOLVE) tile_evolve_one<DIM, BLOCK>(v, c, FOLD_CTA_MIN_LIGHT, smem_raw, ts);
    }
}

}  // namespace
}  // namespace rdb
