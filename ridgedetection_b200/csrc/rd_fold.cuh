// rd_fold.cuh -- exact, parallel evaluation of a left-to-right FP32 sum.
//
// The evolve step of the reference forms every centroid sum as
//     s = 0; for i in members (index order): s = fl(s + x_i)
// (rd/cpu/brute_force/evolve.hpp:71-74), one rounding per member.  Re-
// associating that sum changes its bits, so the GPU must reproduce the chain.
// A chain of dependent adds runs at one add per FADD latency; this file
// evaluates the SAME chain in parallel, exactly:
//
// While every exact intermediate v_i = s_{i-1} + x_i stays inside the binade
// of s, the rounding grid is fixed: with u = ulp(s), S = s/u (an integer of
// magnitude in [2^23, 2^24)) and y_i = x_i/u (a power-of-two scaling, exact),
//     S_i = S_{i-1} + rint(y_i)
// where rint rounds to the nearest integer -- as long as y_i is not exactly
// halfway between two integers, in which case round-to-nearest-even would
// look at the parity of S_{i-1}.  So a run of terms without such a tie adds
// a plain integer sum to S, runs compose by integer prefix sums, and every
// exact v_i of a run lies within 1 of the range of its rounded prefixes.  A
// run is accepted when that range keeps every v_i inside the binade of s and
// none of its terms is a tie or too large; the first run that is not accepted
// (binade crossing, s = 0, a tie, a non-finite term) is folded with plain
// sequential adds and the evaluation restarts after it.  The result is
// bit-identical to the sequential chain for every input; the parallel path
// only decides how much of the chain can be skipped.
#pragma once

#include "rd_internal.cuh"

namespace rdb {
namespace {

constexpr int FOLD_L = 8;                 // members per lane per chunk
constexpr int FOLD_C = 32 * FOLD_L;       // members per chunk

// The rounding grid of s: S = s/u, scale = 1/u, u; ok when s is a normal float
// whose u = 2^(ef-150) and 1/u are normal too (s = 0 and tiny s are not).
struct FoldGrid {
    int S;
    float scale, u;
    bool ok;
};

__device__ __forceinline__ FoldGrid fold_grid(float s)
{
    FoldGrid g;
    const int bits = __float_as_int(s);
    const int ef = (bits >> 23) & 0xff;
    g.ok = (ef >= 24) && (ef <= 254);
    g.scale = __int_as_float((int)((unsigned)(277 - ef) << 23));
    g.u = __int_as_float((int)((unsigned)(ef - 23) << 23));
    const int mant = (bits & 0x7fffff) | 0x800000;
    g.S = (bits < 0) ? -mant : mant;
    return g;
}

// every v in [S + lo, S + hi] lies inside the binade of S (in units of u)
__device__ __forceinline__ bool fold_in_binade(int S, long long lo, long long hi)
{
    return (S > 0) ? (S + lo >= (1 << 23) && S + hi <= (1 << 24) - 1)
                   : (S + hi <= -(1 << 23) && S + lo >= -((1 << 24) - 1));
}

// One lane's run of m terms on the grid of scale: T = sum of rint(y), the
// range [mn, mx] of its prefix sums (0 included), bad = a tie or |y| >= 2^22.
// Terms j >= m enter as zeros (no effect), so the loop has no branches and
// the terms' independent parts overlap.
template <int L>
__device__ __forceinline__ void fold_run(const float (&x)[L], const int m, const float scale,
                                         int& T, int& mn, int& mx, bool& bad)
{
    constexpr float MAGIC = 12582912.0f;  // 1.5 * 2^23: y + MAGIC rounds y to an integer
    int r[L];
    unsigned b = 0u;
#pragma unroll
    for (int j = 0; j < L; ++j) {
        const float y = __fmul_rn((j < m) ? x[j] : 0.0f, scale);
        const float big = __fadd_rn(y, MAGIC);
        const float d = __fsub_rn(y, __fsub_rn(big, MAGIC));
        b |= (unsigned)(!(fabsf(y) < 4194304.0f)) | (unsigned)(fabsf(d) == 0.5f);
        r[j] = __float_as_int(big) - 0x4B400000;
    }
    T = 0;
    mn = 0;
    mx = 0;
#pragma unroll
    for (int j = 0; j < L; ++j) {
        T += r[j];
        mn = min(mn, T);
        mx = max(mx, T);
    }
    bad = b != 0u;
}

// Folds the chunk held by the warp into s: lane l holds, in order, members
// [l*L, l*L + m) of the chunk in x[0..m).  s is warp-uniform in and out.
template <int L>
__device__ __forceinline__ float fold_chunk(float s, const float (&x)[L], const int m, const int lane)
{
    constexpr unsigned FULLM = 0xffffffffu;
    int pos = 0;
    while (pos < 32) {
        const int act = (lane >= pos) ? m : 0;
        const FoldGrid g = fold_grid(s);
        int T, mn, mx;
        bool bad;
        fold_run<L>(x, act, g.scale, T, mn, mx, bad);
        int incl = T;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(FULLM, incl, o);
            if (lane >= o) incl += y;
        }
        const int excl = incl - T;
        const bool ok = (act == 0) ||
                        (g.ok && !bad &&
                         fold_in_binade(g.S, (long long)excl + mn - 1, (long long)excl + mx + 1));
        const unsigned badm = __ballot_sync(FULLM, !ok);
        const int f = badm ? (__ffs(badm) - 1) : 32;
        // commit lanes pos..f-1 (their terms kept s in the binade of s)
        const int Tc = (f < 32) ? __shfl_sync(FULLM, excl, f & 31) : __shfl_sync(FULLM, incl, 31);
        if (g.ok && f > pos) s = __fmul_rn((float)(g.S + Tc), g.u);
        if (f == 32) break;
        // lane f in plain sequential adds; four lanes when nothing was
        // committed (a small or wandering sum, e.g. right after s = 0)
        const int nseq = (f == pos) ? min(4, 32 - f) : 1;
        for (int q = 0; q < nseq; ++q) {
            const int src = f + q;
            const int mf = __shfl_sync(FULLM, m, src);
#pragma unroll
            for (int j = 0; j < L; ++j) {
                const float xj = __shfl_sync(FULLM, x[j], src);
                if (j < mf) s = __fadd_rn(s, xj);
            }
        }
        pos = f + nseq;
    }
    return s;
}

// Sequential FP32 fold, in list order, of the points P[perm[0..n)] with the
// parallel chunk evaluation above (one warp).  The sum of coordinate d is
// returned in lane d < DIM; bit-identical to folding the members one by one.
// Coordinates of chunk c+1 are in flight while chunk c is folded.
template <int DIM>
__device__ float fold_members_par(const int32_t* __restrict__ perm, const int n,
                                  const float* __restrict__ P, const int lane)
{
    constexpr int L = FOLD_L, C = FOLD_C;
    float xc[DIM][L], xn[DIM][L] = {};
    auto gather = [&](float (&x)[DIM][L], int off) {
        int ix[L];
#pragma unroll
        for (int j = 0; j < L; ++j) {
            const int mm = off + lane * L + j;
            ix[j] = (mm < n) ? perm[mm] : -1;
        }
#pragma unroll
        for (int j = 0; j < L; ++j)
#pragma unroll
            for (int d = 0; d < DIM; ++d) x[d][j] = (ix[j] >= 0) ? P[(int64_t)ix[j] * DIM + d] : 0.0f;
    };
    gather(xc, 0);
    float acc[DIM];
#pragma unroll
    for (int d = 0; d < DIM; ++d) acc[d] = 0.0f;
    for (int off = 0; off < n; off += C) {
        const int m = max(0, min(L, n - off - lane * L));
        if (off + C < n) gather(xn, off + C);
#pragma unroll
        for (int d = 0; d < DIM; ++d) acc[d] = fold_chunk<L>(acc[d], xc[d], m, lane);
#pragma unroll
        for (int d = 0; d < DIM; ++d)
#pragma unroll
            for (int j = 0; j < L; ++j) xc[d][j] = xn[d][j];
    }
    float r = 0.0f;
#pragma unroll
    for (int d = 0; d < DIM; ++d) r = (lane == d) ? acc[d] : r;
    return r;
}

// ---------------------------------------------------------------------------
// CTA-wide fold of one long member list.  In a round, warp w summarises chunk
// cb + w (FOLD_C members) on the rounding grid of the running sum at the
// start of the round: its integer total and the range of its prefixes.  Warp
// d then composes coordinate d's summaries (a prefix sum over the chunks, one
// lane per chunk) and accepts them up to the first that would leave the
// binade (the grid does not change while they stay inside); that chunk is
// folded exactly by the warp holding it (fold_chunk).  Coordinates advance
// independently.  Loads run two rounds ahead: member indices of round r+2 and
// coordinates of round r+1 are in flight while round r is summarised.
// ---------------------------------------------------------------------------
struct FoldSummary {
    int T, lo, hi, ok;
};

template <int W, int DIM>
struct FoldCtaSmem {
    FoldSummary sum[W][DIM];
    float s[DIM];
    int cb[2][DIM];   // chunk cursor, double-buffered by round parity
    int stop[DIM];
};

template <int W, int DIM>
__device__ void fold_members_cta(const int32_t* __restrict__ perm, const int n,
                                 const float* __restrict__ P, FoldCtaSmem<W, DIM>& sm)
{
    static_assert(W <= 32, "one lane per chunk in the composition");
    constexpr unsigned FULLM = 0xffffffffu;
    constexpr int L = FOLD_L, C = FOLD_C;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int nch = (n + C - 1) / C;
    auto load_idx = [&](int (&ix)[L], int ch) {
        const int base = ch * C + lane * L;
#pragma unroll
        for (int j = 0; j < L; ++j) ix[j] = (ch < nch && base + j < n) ? perm[base + j] : -1;
    };
    auto gather = [&](float (&x)[L], int& m, const int (&ix)[L], int ch, int d) {
        m = (ch < nch) ? max(0, min(L, n - (ch * C + lane * L))) : 0;
#pragma unroll
        for (int j = 0; j < L; ++j) x[j] = (ix[j] >= 0) ? P[(int64_t)ix[j] * DIM + d] : 0.0f;
    };
    if (tid < DIM) {
        sm.s[tid] = 0.0f;
        sm.cb[0][tid] = 0;
    }
    float xv[DIM][L], xq[DIM][L];
    int iq[DIM][L];
    int mc[DIM], mq[DIM];
#pragma unroll
    for (int d = 0; d < DIM; ++d) {
        int ix[L];
        load_idx(ix, warp);
        gather(xv[d], mc[d], ix, warp, d);
        load_idx(iq[d], W + warp);
    }
    __syncthreads();
    for (int r = 0;; ++r) {
        const int par = r & 1;
        int cb[DIM];
        bool more = false;
#pragma unroll
        for (int d = 0; d < DIM; ++d) {
            cb[d] = sm.cb[par][d];
            more = more || (cb[d] < nch);
        }
        if (!more) break;
        // coordinates of the next round (indices loaded a round ago), indices
        // of the round after; both assume this round accepts all W chunks
        int iqq[DIM][L];
#pragma unroll
        for (int d = 0; d < DIM; ++d) {
            gather(xq[d], mq[d], iq[d], cb[d] + W + warp, d);
            load_idx(iqq[d], cb[d] + 2 * W + warp);
        }
#pragma unroll
        for (int d = 0; d < DIM; ++d) {
            const FoldGrid g = fold_grid(sm.s[d]);
            int T, mn, mx;
            bool bad;
            fold_run<L>(xv[d], mc[d], g.scale, T, mn, mx, bad);
            int incl = T;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const int y = __shfl_up_sync(FULLM, incl, o);
                if (lane >= o) incl += y;
            }
            const int excl = incl - T;
            int lo = (mc[d] > 0) ? excl + mn - 1 : (1 << 30);
            int hi = (mc[d] > 0) ? excl + mx + 1 : -(1 << 30);
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
                lo = min(lo, __shfl_xor_sync(FULLM, lo, o));
                hi = max(hi, __shfl_xor_sync(FULLM, hi, o));
            }
            const bool allok = __all_sync(FULLM, !(mc[d] > 0 && (bad || !g.ok)));
            if (lane == 31) sm.sum[warp][d] = FoldSummary{incl, lo, hi, allok ? 1 : 0};
        }
        __syncthreads();
        // composition of coordinate d by warp d: lane w takes chunk cb + w
        if (warp < DIM) {
            const int d = warp;
            const float s0 = sm.s[d];
            const FoldGrid g = fold_grid(s0);
            const int navail = min(W, nch - cb[d]);
            const bool have = lane < navail;
            const FoldSummary cs = have ? sm.sum[lane][d] : FoldSummary{0, 0, 0, 1};
            int incl = cs.T;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const int y = __shfl_up_sync(FULLM, incl, o);
                if (lane >= o) incl += y;
            }
            const int excl = incl - cs.T;
            const bool good = !have || (g.ok && cs.ok &&
                                        fold_in_binade(g.S, (long long)excl + cs.lo, (long long)excl + cs.hi));
            const unsigned badm = __ballot_sync(FULLM, !good);
            const int f = badm ? (__ffs(badm) - 1) : 32;   // first rejected chunk
            const int acc = min(f, navail);                 // chunks accepted
            const int Tacc = (acc > 0) ? __shfl_sync(FULLM, incl, acc - 1) : 0;
            if (lane == 0) {
                if (acc > 0) sm.s[d] = __fmul_rn((float)(g.S + Tacc), g.u);
                const int stop = (f < navail) ? f : W;
                sm.stop[d] = stop;
                sm.cb[par ^ 1][d] = cb[d] + ((stop < W) ? stop + 1 : W);
            }
        }
        __syncthreads();
#pragma unroll
        for (int d = 0; d < DIM; ++d) {
            const int st = sm.stop[d];
            if (st < W && warp == st) {
                const float s = fold_chunk<L>(sm.s[d], xv[d], mc[d], lane);
                if (lane == 0) sm.s[d] = s;
            }
            if (st < W) {
                // restart after the exactly folded chunk
                const int nb = cb[d] + st + 1;
                int ix[L];
                load_idx(ix, nb + warp);
                gather(xv[d], mc[d], ix, nb + warp, d);
                load_idx(iq[d], nb + W + warp);
            } else {
#pragma unroll
                for (int j = 0; j < L; ++j) {
                    xv[d][j] = xq[d][j];
                    iq[d][j] = iqq[d][j];
                }
                mc[d] = mq[d];
            }
        }
        __syncthreads();
    }
}

}  // namespace
}  // namespace rdb
