// rd_segfold.cuh -- the left-to-right FP32 sum of a long member list,
// exactly, split into segments that warps fold at the same time.
//
// The evolve step sums every cluster's members in index order with one FP32
// rounding per term (rd/cpu/brute_force/evolve.hpp:71-74).  rd_fold.cuh
// evaluates such a chain exactly: while the running sum s stays inside one
// binade, the terms add as integers on s's rounding grid, so runs of terms can
// be added in one step.  A run can only be summarised once the grid of s at
// its start is known, which makes a CTA-wide evaluation proceed in rounds with
// barriers between them.  Here each warp takes a contiguous segment of the
// list and folds it on its own from a SPECULATIVE start value -- the FP64 sum
// of the members before its segment, rounded to FP32 -- while recording a
// trace of what it did:
//   RUN    terms added as one integer total T on the grid of a given binade,
//          with the range [lo, hi] of the run's prefix sums (rounding margin
//          included) relative to the run's start;
//   EXACT  terms added one rounding at a time (a binade crossing, a tie, a
//          sum too close to zero);
//   ABORT  the trace is full: the rest of the segment is not described.
// One warp then replays the traces in segment order from the exact start.  A
// RUN applies to any start S on the same grid whose prefix range
// [S + lo, S + hi] stays inside the binade (the per-term roundings are then
// the same, because rounding on a fixed grid depends only on the term), so it
// is added in one step; EXACT terms are folded one by one from the exact
// value; a RUN that does not apply, or an ABORT, makes the replay fold the rest
// of that segment exactly.  When the exact start equals the speculative one
// bit for bit, the segment's speculative result is taken as it is.  The result
// is bit-identical to the serial chain for every input: speculation only
// decides how much work the replay can skip.  The FP64 estimate is close to
// the FP32 running sum (its error is a few ulps of the sum per thousands of
// terms), so nearly every RUN applies.
#pragma once

#include "rd_fold.cuh"

namespace rdb {
namespace {

constexpr int SEG_TR = 6;                 // trace entries per (segment, coordinate)

// Where the members of a list live.  IdxSrc: member i is point mem[i] of P
// (DIM floats per point), so a load is an index load and a dependent
// coordinate load.  RowSrc: member i is row i of a grouped copy (PadDim<DIM>
// floats per row, DIM 3 as float4), laid out by the stable scatter of the
// lockstep passes, so a list is one contiguous stream.  Both give the same
// values in the same order.
template <int DIM>
struct IdxSrc {
    const int32_t* __restrict__ mem;
    const float* __restrict__ P;
    // members off + j, j < m, into x[.][j] (zeros beyond m)
    template <int L>
    __device__ __forceinline__ void load_run(int off, int m, float (&x)[DIM][L]) const
    {
        int ix[L];
#pragma unroll
        for (int j = 0; j < L; ++j) ix[j] = (j < m) ? mem[off + j] : -1;
#pragma unroll
        for (int j = 0; j < L; ++j)
#pragma unroll
            for (int d = 0; d < DIM; ++d) x[d][j] = (ix[j] >= 0) ? P[(int64_t)ix[j] * DIM + d] : 0.0f;
    }
    template <int L>
    __device__ __forceinline__ void load_run1(int off, int m, int d, float (&x)[L]) const
    {
        int ix[L];
#pragma unroll
        for (int j = 0; j < L; ++j) ix[j] = (j < m) ? mem[off + j] : -1;
#pragma unroll
        for (int j = 0; j < L; ++j) x[j] = (ix[j] >= 0) ? P[(int64_t)ix[j] * DIM + d] : 0.0f;
    }
};

template <int DIM>
struct RowSrc {
    const float* __restrict__ rows;
    __device__ __forceinline__ void load_row(int i, float (&x)[DIM]) const
    {
        if constexpr (PadDim<DIM>::v == 4) {
            const float4 t = reinterpret_cast<const float4*>(rows)[i];
            x[0] = t.x;
            if constexpr (DIM > 1) x[1] = t.y;
            if constexpr (DIM > 2) x[2] = t.z;
            if constexpr (DIM > 3) x[3] = t.w;
        } else if constexpr (DIM == 2) {
            const float2 t = reinterpret_cast<const float2*>(rows)[i];
            x[0] = t.x;
            x[1] = t.y;
        } else {
#pragma unroll
            for (int d = 0; d < DIM; ++d) x[d] = rows[(int64_t)i * PadDim<DIM>::v + d];
        }
    }
    template <int L>
    __device__ __forceinline__ void load_run(int off, int m, float (&x)[DIM][L]) const
    {
#pragma unroll
        for (int j = 0; j < L; ++j) {
            float r[DIM];
#pragma unroll
            for (int d = 0; d < DIM; ++d) r[d] = 0.0f;
            if (j < m) load_row(off + j, r);
#pragma unroll
            for (int d = 0; d < DIM; ++d) x[d][j] = r[d];
        }
    }
    template <int L>
    __device__ __forceinline__ void load_run1(int off, int m, int d, float (&x)[L]) const
    {
#pragma unroll
        for (int j = 0; j < L; ++j)
            x[j] = (j < m) ? rows[(int64_t)(off + j) * PadDim<DIM>::v + d] : 0.0f;
    }
};

enum : int { SK_RUN = 0, SK_EXACT = 1, SK_ABORT = 2 };

struct SegEntry {
    int kg;       // kind | grid bits of the running sum (sign and exponent)
    int T;        // RUN: integer total on that grid
    int lo, hi;   // RUN: prefix range relative to the run's start
    int m;        // members covered
    int pad[3];
};

struct alignas(16) SegTrace {
    float start;  // speculative start value
    float fin;    // speculative end value
    int n;        // entries
    int pad;
    SegEntry e[SEG_TR];
};

__device__ __forceinline__ int fold_grid_bits(float s) { return __float_as_int(s) & (int)0xFF800000u; }

// Trace state of one coordinate, warp-uniform; the entry being built stays in
// registers until the next one starts.
struct SegRec {
    int kind;     // -1: none
    int grid, T, lo, hi, m;
    int n;        // entries written
};

__device__ __forceinline__ void segrec_init(SegRec& r)
{
    r.kind = -1;
    r.grid = r.T = r.lo = r.hi = r.m = 0;
    r.n = 0;
}

// writes the entry being built (lane 0); the last slot becomes an ABORT
__device__ __forceinline__ void segrec_flush(SegRec& r, SegTrace& tr, const int lane)
{
    if (r.kind < 0 || r.n >= SEG_TR) return;
    if (lane == 0) {
        SegEntry en;
        en.kg = (r.n == SEG_TR - 1) ? SK_ABORT : (r.kind | r.grid);
        en.T = r.T;
        en.lo = r.lo;
        en.hi = r.hi;
        en.m = r.m;
        tr.e[r.n] = en;
    }
    ++r.n;
    r.kind = -1;
}

__device__ __forceinline__ void segrec_run(SegRec& r, SegTrace& tr, int grid, int T, int lo, int hi,
                                           int m, const int lane)
{
    if (r.n >= SEG_TR) return;
    if (r.kind == SK_RUN && r.grid == grid) {
        r.lo = min(r.lo, r.T + lo);
        r.hi = max(r.hi, r.T + hi);
        r.T += T;
        r.m += m;
        return;
    }
    segrec_flush(r, tr, lane);
    r.kind = SK_RUN;
    r.grid = grid;
    r.T = T;
    r.lo = lo;
    r.hi = hi;
    r.m = m;
}

__device__ __forceinline__ void segrec_exact(SegRec& r, SegTrace& tr, int m, const int lane)
{
    if (r.n >= SEG_TR || m == 0) return;
    if (r.kind == SK_EXACT) {
        r.m += m;
        return;
    }
    segrec_flush(r, tr, lane);
    r.kind = SK_EXACT;
    r.m = m;
}

// fold_chunk (rd_fold.cuh) with a trace: lane l holds members [l*L, l*L + m)
// of a chunk of mtot members in x; s is warp-uniform in and out.
template <int L>
__device__ __forceinline__ float fold_chunk_traced(float s, const float (&x)[L], const int m,
                                                   const int mtot, const int lane, SegRec& rec,
                                                   SegTrace& tr)
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
        const int Tc = (f < 32) ? __shfl_sync(FULLM, excl, f & 31) : __shfl_sync(FULLM, incl, 31);
        // the run committed: lanes [pos, f) (those holding members)
        const bool inrun = lane >= pos && lane < f && act > 0;
        int lo = inrun ? excl + mn - 1 : (1 << 30);
        int hi = inrun ? excl + mx + 1 : -(1 << 30);
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            lo = min(lo, __shfl_xor_sync(FULLM, lo, o));
            hi = max(hi, __shfl_xor_sync(FULLM, hi, o));
        }
        if (g.ok && f > pos && lo <= hi) {
            const int mm = max(0, min(mtot - pos * L, (f - pos) * L));
            segrec_run(rec, tr, fold_grid_bits(s), Tc, lo, hi, mm, lane);
            s = __fmul_rn((float)(g.S + Tc), g.u);
        }
        if (f == 32) break;
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
        segrec_exact(rec, tr, max(0, min(mtot - f * L, nseq * L)), lane);
        pos = f + nseq;
    }
    return s;
}

// One warp folds members [b, e) of the list mem (coordinates of P, DIM per
// point) from the start values s[d] (warp-uniform), recording the trace of
// coordinate d in tr[d]; tr[d].start/fin/n are written by lane 0.  The next
// chunk's indices and coordinates are loaded while a chunk is folded.
template <int DIM, class Src>
__device__ void warp_fold_traced_src(const Src& src, const int b, const int e, float (&s)[DIM],
                                     SegTrace* tr, const int lane)
{
    constexpr int L = FOLD_L, C = FOLD_C;
    SegRec rec[DIM];
#pragma unroll
    for (int d = 0; d < DIM; ++d) {
        segrec_init(rec[d]);
        if (lane == 0) tr[d].start = s[d];
    }
    float xn[DIM][L];
    int mn_ = 0;
    auto gather = [&](float (&x)[DIM][L], int& m, int off) {
        const int mtot = min(C, e - off);
        m = (off < e) ? max(0, min(L, mtot - lane * L)) : 0;
        src.template load_run<L>(off + lane * L, m, x);
    };
    if (b < e) gather(xn, mn_, b);
    for (int off = b; off < e; off += C) {
        float xc[DIM][L];
        const int mc = mn_;
        const int mtot = min(C, e - off);
#pragma unroll
        for (int d = 0; d < DIM; ++d)
#pragma unroll
            for (int j = 0; j < L; ++j) xc[d][j] = xn[d][j];
        if (off + C < e) gather(xn, mn_, off + C);
#pragma unroll
        for (int d = 0; d < DIM; ++d)
            s[d] = fold_chunk_traced<L>(s[d], xc[d], mc, mtot, lane, rec[d], tr[d]);
    }
#pragma unroll
    for (int d = 0; d < DIM; ++d) {
        segrec_flush(rec[d], tr[d], lane);
        if (lane == 0) {
            tr[d].n = min(rec[d].n, SEG_TR);
            tr[d].fin = s[d];
        }
    }
}

template <int DIM>
__device__ __forceinline__ void warp_fold_traced(const int32_t* __restrict__ mem, const int b,
                                                 const int e, const float* __restrict__ P,
                                                 float (&s)[DIM], SegTrace* tr, const int lane)
{
    warp_fold_traced_src<DIM>(IdxSrc<DIM>{mem, P}, b, e, s, tr, lane);
}

// One warp folds members [from, to) of the list exactly (coordinate d) into
// the warp-uniform s, a chunk of FOLD_C members at a time; the next chunk's
// indices and coordinates are in flight while a chunk is folded.
template <int DIM, class Src>
__device__ float fold_range_exact(const Src& src, int from, const int to, const int d, float s,
                                  const int lane)
{
    constexpr int L = FOLD_L, C = FOLD_C;
    auto gather = [&](float (&x)[L], int& m, int off) {
        const int mtot = min(C, to - off);
        m = max(0, min(L, mtot - lane * L));
        src.template load_run1<L>(off + lane * L, m, d, x);
    };
    float xn[L];
    int mn = 0;
    if (from < to) gather(xn, mn, from);
    for (; from < to; from += C) {
        float xc[L];
#pragma unroll
        for (int j = 0; j < L; ++j) xc[j] = xn[j];
        const int mc = mn;
        if (from + C < to) gather(xn, mn, from + C);
        s = fold_chunk<L>(s, xc, mc, lane);
    }
    return s;
}

// The exact value after segment [b, e) of the list for the exact start s,
// from the segment's trace (which may live in another CTA's shared memory).
template <int DIM, class Src>
__device__ float replay_segment_src(const SegTrace& tr, const Src& src, const int b, const int e,
                                    const int d, float s, const int lane)
{
    if (__float_as_int(s) == __float_as_int(tr.start)) return tr.fin;
    const int n = tr.n;
    int off = b;
    for (int t = 0; t < n; ++t) {
        const SegEntry en = tr.e[t];
        const int kind = en.kg & 3;
        if (kind == SK_RUN) {
            const FoldGrid g = fold_grid(s);
            if (g.ok && fold_grid_bits(s) == (en.kg & ~3) && fold_in_binade(g.S, en.lo, en.hi)) {
                s = __fmul_rn((float)(g.S + en.T), g.u);
                off += en.m;
                continue;
            }
            return fold_range_exact<DIM>(src, off, e, d, s, lane);
        }
        if (kind == SK_EXACT) {
            s = fold_range_exact<DIM>(src, off, off + en.m, d, s, lane);
            off += en.m;
            continue;
        }
        return fold_range_exact<DIM>(src, off, e, d, s, lane);   // ABORT
    }
    return s;
}

template <int DIM>
__device__ __forceinline__ float replay_segment(const SegTrace& tr, const int32_t* __restrict__ mem,
                                                const int b, const int e,
                                                const float* __restrict__ P, const int d, float s,
                                                const int lane)
{
    return replay_segment_src<DIM>(tr, IdxSrc<DIM>{mem, P}, b, e, d, s, lane);
}

// FP64 sum of members [b, e) of the list, by one warp; every lane holds it.
// SUM64_U members per lane are gathered before any of them is added, so the
// dependent index-then-coordinate loads of a step overlap instead of queueing
// behind the add chain.
constexpr int SUM64_U = 8;

template <int DIM>
__device__ void warp_sum64_add(const IdxSrc<DIM>& src, const int b, const int e,
                               double (&acc)[DIM], const int lane)
{
    constexpr int U = SUM64_U;
    for (int i0 = b; i0 < e; i0 += 32 * U) {
        int ix[U];
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const int i = i0 + u * 32 + lane;
            ix[u] = (i < e) ? src.mem[i] : -1;
        }
        float x[U][DIM];
#pragma unroll
        for (int u = 0; u < U; ++u)
#pragma unroll
            for (int d = 0; d < DIM; ++d)
                x[u][d] = (ix[u] >= 0) ? src.P[(int64_t)ix[u] * DIM + d] : 0.0f;
#pragma unroll
        for (int u = 0; u < U; ++u)
#pragma unroll
            for (int d = 0; d < DIM; ++d) acc[d] += (double)x[u][d];
    }
}

template <int DIM>
__device__ void warp_sum64_add(const RowSrc<DIM>& src, const int b, const int e,
                               double (&acc)[DIM], const int lane)
{
    constexpr int U = SUM64_U;
    for (int i0 = b; i0 < e; i0 += 32 * U) {
        float x[U][DIM];
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const int i = i0 + u * 32 + lane;
#pragma unroll
            for (int d = 0; d < DIM; ++d) x[u][d] = 0.0f;
            if (i < e) src.load_row(i, x[u]);
        }
#pragma unroll
        for (int u = 0; u < U; ++u)
#pragma unroll
            for (int d = 0; d < DIM; ++d) acc[d] += (double)x[u][d];
    }
}

template <int DIM, class Src>
__device__ void warp_sum64_src(const Src& src, const int b, const int e, double (&acc)[DIM],
                               const int lane)
{
#pragma unroll
    for (int d = 0; d < DIM; ++d) acc[d] = 0.0;
    warp_sum64_add<DIM>(src, b, e, acc, lane);
#pragma unroll
    for (int d = 0; d < DIM; ++d)
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) acc[d] += __shfl_xor_sync(0xffffffffu, acc[d], o);
}

template <int DIM>
__device__ __forceinline__ void warp_sum64(const int32_t* __restrict__ mem, const int b,
                                           const int e, const float* __restrict__ P,
                                           double (&acc)[DIM], const int lane)
{
    warp_sum64_src<DIM>(IdxSrc<DIM>{mem, P}, b, e, acc, lane);
}

// ---------------------------------------------------------------------------
// One CTA (W warps): the list mem[0..n) in W segments; the exact sums of the
// DIM coordinates end up in sm.out.  Two CTA barriers and one composition
// warp per coordinate.
// ---------------------------------------------------------------------------
template <int W, int DIM>
struct SegFoldSmem {
    double part[W][DIM];
    SegTrace tr[W][DIM];
    float out[DIM];
};

template <int W, int DIM, class Src>
__device__ void fold_members_seg_src(const Src& src, const int n, SegFoldSmem<W, DIM>& sm)
{
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int b = (int)(((int64_t)warp * n) / W), e = (int)(((int64_t)(warp + 1) * n) / W);
    double acc[DIM];
    warp_sum64_src<DIM>(src, b, e, acc, lane);
    if (lane == 0)
#pragma unroll
        for (int d = 0; d < DIM; ++d) sm.part[warp][d] = acc[d];
    __syncthreads();
    float s[DIM];
#pragma unroll
    for (int d = 0; d < DIM; ++d) {
        double est = 0.0;
        for (int w = 0; w < warp; ++w) est += sm.part[w][d];
        s[d] = (warp == 0) ? 0.0f : (float)est;
    }
    warp_fold_traced_src<DIM>(src, b, e, s, sm.tr[warp], lane);
    __syncthreads();
    if (warp < DIM) {
        const int d = warp;
        float x = sm.tr[0][d].fin;   // segment 0 started exactly at 0
        for (int w = 1; w < W; ++w) {
            const int bw = (int)(((int64_t)w * n) / W), ew = (int)(((int64_t)(w + 1) * n) / W);
            x = replay_segment_src<DIM>(sm.tr[w][d], src, bw, ew, d, x, lane);
        }
        if (lane == 0) sm.out[d] = x;
    }
    __syncthreads();
}

template <int W, int DIM>
__device__ __forceinline__ void fold_members_seg(const int32_t* __restrict__ mem, const int n,
                                                 const float* __restrict__ P,
                                                 SegFoldSmem<W, DIM>& sm)
{
    fold_members_seg_src<W, DIM>(IdxSrc<DIM>{mem, P}, n, sm);
}

}  // namespace
}  // namespace rdb
