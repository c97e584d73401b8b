// rd_grid.cuh -- hashed uniform grid helpers and the in-order decimation scan,
// shared by the engine kernels (rd_kernels.cu) and the allocation-free
// decimation entry point (rd_noalloc.cu).
#pragma once

#include "rd_internal.cuh"

namespace rdb {
namespace {

constexpr unsigned FULL = 0xffffffffu;

template <int DIM>
struct Pow3 { static constexpr int v = 3 * Pow3<DIM - 1>::v; };
template <>
struct Pow3<0> { static constexpr int v = 1; };

__device__ __forceinline__ int cell_of(float x, double inv)
{
    double c = floor((double)x * inv);
    c = fmin(fmax(c, -1073741824.0), 1073741823.0);
    return (int)c;
}

template <int DIM>
__device__ __forceinline__ uint32_t cell_hash(const int* c)
{
    uint32_t h = 2166136261u;
#pragma unroll
    for (int d = 0; d < DIM; ++d) h = (h ^ (uint32_t)c[d]) * 16777619u;
    return h ^ (h >> 15);
}

// barrier `id` (1..15; 0 is __syncthreads) over `n` threads, whole warps
__device__ __forceinline__ void named_bar_sync(int id, int n)
{
    asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(n) : "memory");
}

// offset o in [0, 3^DIM) -> neighbour cell; o == (3^DIM-1)/2 is the home cell
template <int DIM>
__device__ __forceinline__ void neighbour_cell(const int* cc, int o, int* out)
{
#pragma unroll
    for (int d = 0; d < DIM; ++d) {
        out[d] = cc[d] + (o % 3) - 1;
        o /= 3;
    }
}

// In-order decimation of X[0..total) (rd/cpu/brute_force/decimate.hpp:41-81, or
// :85-127 when nocopy): leaves alive[i] = 1 for the survivors.  Scratch: cell
// (total*DIM), alive, c1, c2, items (total each), bstart (hmask+2).  All
// threads of the block call it.
template <int DIM, int BLOCK>
__device__ void decimate_scan(const float* X, const int total, const float r2, const int nocopy,
                              int32_t* cell, int32_t* alive, int32_t* c1, int32_t* c2,
                              int32_t* items, int32_t* bstart, const uint32_t hmask, int32_t* err)
{
    constexpr int NB = Pow3<DIM>::v;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const float rsq = sqr_rn(r2);
    const float rsq4 = __fmul_rn(4.0f, rsq);
    const double inv = 1.0 / (2.0 * (double)r2 * (1.0 + 1.0 / 1024.0));
    for (int h = tid; h <= (int)hmask + 1; h += BLOCK) bstart[h] = 0;
    __syncthreads();
    // cells and bucket counts
    for (int i = tid; i < total; i += BLOCK) {
        int cc[DIM];
#pragma unroll
        for (int d = 0; d < DIM; ++d) {
            cc[d] = cell_of(X[(int64_t)i * DIM + d], inv);
            cell[(int64_t)i * DIM + d] = cc[d];
        }
        atomicAdd(&bstart[(cell_hash<DIM>(cc) & hmask) + 1], 1);
        alive[i] = 1;
    }
    __syncthreads();
    // exclusive prefix over buckets (single warp, sequential carry)
    if (warp == 0) {
        int carry = 0;
        for (int h0 = 0; h0 <= (int)hmask + 1; h0 += 32) {
            const int h = h0 + lane;
            int x = (h <= (int)hmask + 1) ? bstart[h] : 0;
            int incl = x;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const int y = __shfl_up_sync(FULL, incl, o);
                if (lane >= o) incl += y;
            }
            if (h <= (int)hmask + 1) bstart[h] = carry + incl;
            carry += __shfl_sync(FULL, incl, 31);
        }
    }
    __syncthreads();
    // fill buckets (member order inside a bucket does not matter: counts only)
    for (int i = tid; i < total; i += BLOCK) {
        int cc[DIM];
#pragma unroll
        for (int d = 0; d < DIM; ++d) cc[d] = cell[(int64_t)i * DIM + d];
        const uint32_t b = cell_hash<DIM>(cc) & hmask;
        const int slot = atomicAdd(&bstart[b], 1);
        items[slot] = i;
    }
    __syncthreads();
    // bstart[b] now holds the end of bucket b; start of b is bstart[b-1] (0 for b = 0)
    auto bucket_range = [&](uint32_t b, int& lo, int& hi) {
        lo = (b == 0) ? 0 : bstart[b - 1];
        hi = bstart[b];
    };
    // initial counts
    for (int i = tid; i < total; i += BLOCK) {
        float p[DIM];
        int cc[DIM];
#pragma unroll
        for (int d = 0; d < DIM; ++d) {
            p[d] = X[(int64_t)i * DIM + d];
            cc[d] = cell[(int64_t)i * DIM + d];
        }
        int n1 = 0, n2 = 0;
        for (int o = 0; o < NB; ++o) {
            int nc[DIM];
            neighbour_cell<DIM>(cc, o, nc);
            int lo, hi;
            bucket_range(cell_hash<DIM>(nc) & hmask, lo, hi);
            for (int t = lo; t < hi; ++t) {
                const int q = items[t];
                bool same = true;
#pragma unroll
                for (int d = 0; d < DIM; ++d) same = same && (cell[(int64_t)q * DIM + d] == nc[d]);
                if (!same) continue;
                float s[DIM];
#pragma unroll
                for (int d = 0; d < DIM; ++d) s[d] = X[(int64_t)q * DIM + d];
                const float sq = sqdist_exact<DIM>(p, s);
                n1 += (sq <= rsq);
                n2 += (sq <= rsq4);
            }
        }
        c1[i] = n1;
        c2[i] = n2;
    }
    __syncthreads();
    // sequential in-order scan (warp 0)
    if (warp == 0) {
        int cnt = total, left = -1, guard = 0;
        bool stop = false;
        while (left != cnt && cnt > 3 && !stop) {
            if (++guard > total + 2) { if (lane == 0) atomicOr(err, ERRB_DEC_CAP); break; }
            left = cnt;
            int i = 0;
            while (i < total) {
                const int w = i + lane;
                const bool pred = (w < total) && alive[w] && (c1[w] >= 4 || c2[w] < 3);
                const unsigned bal = __ballot_sync(FULL, pred);
                if (bal == 0) { i += 32; continue; }
                const int j = i + __ffs(bal) - 1;
                if (nocopy && cnt - 1 < 3) { stop = true; break; }
                if (lane == 0) alive[j] = 0;
                --cnt;
                // decrement the counts of j's neighbours
                float p[DIM];
                int cc[DIM];
#pragma unroll
                for (int d = 0; d < DIM; ++d) {
                    p[d] = X[(int64_t)j * DIM + d];
                    cc[d] = cell[(int64_t)j * DIM + d];
                }
                for (int o = 0; o < NB; ++o) {
                    int nc[DIM];
                    neighbour_cell<DIM>(cc, o, nc);
                    int lo, hi;
                    bucket_range(cell_hash<DIM>(nc) & hmask, lo, hi);
                    for (int t = lo + lane; t < hi; t += 32) {
                        const int q = items[t];
                        if (q == j) continue;
                        bool same = true;
#pragma unroll
                        for (int d = 0; d < DIM; ++d) same = same && (cell[(int64_t)q * DIM + d] == nc[d]);
                        if (!same) continue;
                        float s[DIM];
#pragma unroll
                        for (int d = 0; d < DIM; ++d) s[d] = X[(int64_t)q * DIM + d];
                        const float sq = sqdist_exact<DIM>(p, s);
                        if (sq <= rsq4) c2[q] -= 1;   // distinct q per lane: no race
                        if (sq <= rsq) c1[q] -= 1;
                    }
                }
                __syncwarp();
                if (!nocopy && cnt < 3) break;
                i = j + 1;
            }
            if (!nocopy && cnt < 3) break;
        }
    }
    __syncthreads();
}


// Visits every point q != i within 2*r2 of point i of X (bucketed by the
// counting sort in items/bstart, cells in cell): f(q, within_r2).
template <int DIM, class F>
__device__ __forceinline__ void dec_for_neighbours(const int i, const float* X,
                                                   const int32_t* cell, const int32_t* items,
                                                   const int32_t* bstart, const uint32_t hmask,
                                                   const float rsq, const float rsq4, F&& f)
{
    constexpr int NB = Pow3<DIM>::v;
    float p[DIM];
    int cc[DIM];
#pragma unroll
    for (int d = 0; d < DIM; ++d) {
        p[d] = X[(int64_t)i * DIM + d];
        cc[d] = cell[(int64_t)i * DIM + d];
    }
    for (int o = 0; o < NB; ++o) {
        int nc[DIM];
        neighbour_cell<DIM>(cc, o, nc);
        const uint32_t b = cell_hash<DIM>(nc) & hmask;
        const int lo = (b == 0) ? 0 : bstart[b - 1];
        const int hi = bstart[b];
        for (int t = lo; t < hi; ++t) {
            const int q = items[t];
            if (q == i) continue;
            bool same = true;
#pragma unroll
            for (int d = 0; d < DIM; ++d) same = same && (cell[(int64_t)q * DIM + d] == nc[d]);
            if (!same) continue;
            float s[DIM];
#pragma unroll
            for (int d = 0; d < DIM; ++d) s[d] = X[(int64_t)q * DIM + d];
            const float sq = sqdist_exact<DIM>(p, s);
            if (sq <= rsq4) f(q, sq <= rsq);
        }
    }
}

// Passes of the in-order decimation, resolved in parallel rounds (exact).
// In one pass the reference visits the alive points in order and removes
// point i when, at that moment, c1 >= 4 or c2 < 3 (alive points within r2 /
// 2*r2, self included); a removal lowers the counts of its neighbours.  At
// i's turn only its EARLIER neighbours can have been removed in this pass, and
// counts only fall, so with rem = earlier neighbours known removed and und =
// earlier neighbours still undecided:
//   c1 at i's turn lies in [c1 - rem1 - und1, c1 - rem1], c2 likewise;
//   i is surely removed when c1 - rem1 - und1 >= 4 or c2 - rem2 < 3,
//   surely kept when c1 - rem1 < 4 and c2 - rem2 - und2 >= 3.
// Rounds decide every point they can until none is undecided; the lowest
// undecided point always has und = 0, so each round decides at least one.
// The reference also stops removing once fewer than 3 points would remain
// (decimate.hpp:62-80 breaks the pass, decimateNoCopy keeps the point); a pass
// whose removals leave at least 3 points never meets that rule, and a pass
// that would leave fewer is not applied: *fallback is set and the caller
// finishes with the sequential scan from the state before that pass.
// State per point st[i]: 0 dead, 1 alive (undecided in a pass), 2 kept in
// this pass, 3 removed in this pass; counts c1/c2 of alive points are exact
// between passes.  Returns the alive count.  All threads of the block call it.
// tally (optional): tally[0] += passes resolved, tally[1] += rounds they took.
template <int BLOCK, class CT, class ST>
__device__ int decimate_round_passes(const int total, int cnt, CT* c1, CT* c2, ST* st_,
                                     const int32_t* nb_off, const int32_t* nb, int* fallback,
                                     int32_t* err, int32_t* tally = nullptr)
{
    volatile ST* st = st_;
    const int tid = threadIdx.x;
    *fallback = 0;
    int guard = 0;
    while (cnt > 3) {
        if (++guard > total + 2) {
            if (tid == 0) atomicOr(err, ERRB_DEC_CAP);
            break;
        }
        // one pass, in rounds
        for (int round = 0;; ++round) {
            int und_left = 0;
            for (int i = tid; i < total; i += BLOCK) {
                if (st[i] != 1) continue;
                int rem1 = 0, und1 = 0, rem2 = 0, und2 = 0;
                const int e1 = nb_off[i + 1];
                for (int t = nb_off[i]; t < e1; ++t) {
                    const int e = nb[t];
                    const int q = e & 0x7fffffff;
                    if (q >= i) continue;
                    const int sq = st[q];
                    const int w1 = (e < 0) ? 1 : 0;
                    rem2 += (sq == 3);
                    rem1 += (sq == 3) & w1;
                    und2 += (sq == 1);
                    und1 += (sq == 1) & w1;
                }
                const int a = (int)c1[i] - rem1, b = (int)c2[i] - rem2;
                if (a - und1 >= 4 || b < 3) st[i] = 3;
                else if (a < 4 && b - und2 >= 3) st[i] = 2;
                else und_left = 1;
            }
            if (tally && tid == 0) atomicAdd(&tally[1], 1);
            if (!__syncthreads_or(und_left)) break;
            if (round > total) {   // cannot happen: every round decides a point
                if (tid == 0) atomicOr(err, ERRB_DEC_CAP);
                break;
            }
        }
        __shared__ int s_removed;
        if (tid == 0) {
            s_removed = 0;
            if (tally) atomicAdd(&tally[0], 1);
        }
        __syncthreads();
        int mine = 0;
        for (int i = tid; i < total; i += BLOCK) mine += (st[i] == 3);
        if (mine) atomicAdd(&s_removed, mine);
        __syncthreads();
        const int removed = s_removed;
        const bool apply = removed > 0 && cnt - removed >= 3;
        for (int i = tid; i < total; i += BLOCK) {
            const int v = st[i];
            if (v == 3) st[i] = apply ? 0 : 1;
            else if (v == 2) st[i] = 1;
        }
        __syncthreads();
        if (removed == 0) break;            // a pass that changed nothing ends the loop
        if (!apply) {                       // the minimum-count rule may act
            *fallback = 1;
            break;
        }
        cnt -= removed;
        // exact counts of the alive points for the next pass
        for (int i = tid; i < total; i += BLOCK) {
            if (st[i] != 1) continue;
            int n1 = 1, n2 = 1;
            const int e1 = nb_off[i + 1];
            for (int t = nb_off[i]; t < e1; ++t) {
                const int e = nb[t];
                if (st[e & 0x7fffffff] == 1) {
                    ++n2;
                    n1 += (e < 0) ? 1 : 0;
                }
            }
            c1[i] = (CT)n1;
            c2[i] = (CT)n2;
        }
        __syncthreads();
    }
    return cnt;
}

// Same decimation as decimate_scan, faster for large sets: every point's
// neighbours within 2*r2 are listed once (CSR in nb_off/nb, the sign bit
// marking "also within r2"), so a removal decrements its neighbours' counts
// with one coalesced read of its list; counts and alive flags live in shared
// memory (smem, 5 bytes per point) when total <= smem_max.  Falls back to
// decimate_scan when the lists do not fit in nb_cap.  alive[] (global)
// receives the survivors either way.
template <int DIM, int BLOCK>
__device__ void decimate_scan_lists(const float* X, const int total, const float r2,
                                    const int nocopy, int32_t* cell, int32_t* alive, int32_t* c1g,
                                    int32_t* c2g, int32_t* items, int32_t* bstart,
                                    const uint32_t hmask, int32_t* nb_off, int32_t* nb,
                                    const int64_t nb_cap, unsigned char* smem, const int smem_max,
                                    int32_t* err, const int prepared = 0, int32_t* tally = nullptr)
{
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const float rsq = sqr_rn(r2);
    const float rsq4 = __fmul_rn(4.0f, rsq);
    const double inv = 1.0 / (2.0 * (double)r2 * (1.0 + 1.0 / 1024.0));
    const bool in_smem = total <= smem_max;
    int16_t* c1s = reinterpret_cast<int16_t*>(smem);
    int16_t* c2s = c1s + smem_max;
    unsigned char* as = reinterpret_cast<unsigned char*>(c2s + smem_max);
    // candidate bitmap (alive and removable right now), 16-byte aligned after the flags
    uint32_t* cand = reinterpret_cast<uint32_t*>(
        smem + ((2 * sizeof(int16_t) * smem_max + smem_max + 15) / 16) * 16);
    __shared__ int s_carry, s_overflow;
    __shared__ int s_w[BLOCK / 32];

    if (prepared) {  // buckets, counts and lists were built by the GPU-wide kernels
        for (int i = tid; i < total; i += BLOCK) {
            if (in_smem) {
                c1s[i] = (int16_t)c1g[i];
                c2s[i] = (int16_t)c2g[i];
                as[i] = 1;
            }
            alive[i] = 1;
        }
        __syncthreads();
    } else {
    for (int h = tid; h <= (int)hmask + 1; h += BLOCK) bstart[h] = 0;
    if (tid == 0) { s_carry = 0; s_overflow = 0; }
    __syncthreads();
    for (int i = tid; i < total; i += BLOCK) {
        int cc[DIM];
#pragma unroll
        for (int d = 0; d < DIM; ++d) {
            cc[d] = cell_of(X[(int64_t)i * DIM + d], inv);
            cell[(int64_t)i * DIM + d] = cc[d];
        }
        atomicAdd(&bstart[(cell_hash<DIM>(cc) & hmask) + 1], 1);
    }
    __syncthreads();
    if (warp == 0) {
        int carry = 0;
        for (int h0 = 0; h0 <= (int)hmask + 1; h0 += 32) {
            const int h = h0 + lane;
            int x = (h <= (int)hmask + 1) ? bstart[h] : 0;
            int incl = x;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const int y = __shfl_up_sync(FULL, incl, o);
                if (lane >= o) incl += y;
            }
            if (h <= (int)hmask + 1) bstart[h] = carry + incl;
            carry += __shfl_sync(FULL, incl, 31);
        }
    }
    __syncthreads();
    for (int i = tid; i < total; i += BLOCK) {
        int cc[DIM];
#pragma unroll
        for (int d = 0; d < DIM; ++d) cc[d] = cell[(int64_t)i * DIM + d];
        const int slot = atomicAdd(&bstart[cell_hash<DIM>(cc) & hmask], 1);
        items[slot] = i;
    }
    __syncthreads();
    auto for_neighbours = [&](int i, auto&& f) {
        dec_for_neighbours<DIM>(i, X, cell, items, bstart, hmask, rsq, rsq4, f);
    };
    // counts (self included) and list lengths
    for (int i = tid; i < total; i += BLOCK) {
        int n1 = 1, n2 = 1;
        for_neighbours(i, [&](int, bool w1) { ++n2; n1 += w1; });
        if (in_smem) {
            c1s[i] = (int16_t)n1;
            c2s[i] = (int16_t)n2;
            as[i] = 1;
        } else {
            c1g[i] = n1;
            c2g[i] = n2;
        }
        alive[i] = 1;
        nb_off[i] = n2 - 1;
    }
    __syncthreads();
    // exclusive prefix of list lengths
    for (int i0 = 0; i0 < total; i0 += BLOCK) {
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
        for (int w = 0; w < BLOCK / 32; ++w) {
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
        s_overflow = (int64_t)s_carry > nb_cap;
    }
    __syncthreads();
    if (s_overflow) {  // lists do not fit: bucket-walk version
        decimate_scan<DIM, BLOCK>(X, total, r2, nocopy, cell, alive, c1g, c2g, items, bstart, hmask,
                                  err);
        return;
    }
    for (int i = tid; i < total; i += BLOCK) {
        int k = nb_off[i];
        for_neighbours(i, [&](int q, bool w1) { nb[k++] = w1 ? (q | (int)0x80000000) : q; });
    }
    __syncthreads();
    }
    // passes in parallel rounds while the minimum-count rule cannot act
    __shared__ int s_alive, s_fallback;
    {
        int fb = 0;
        const int left = in_smem
            ? decimate_round_passes<BLOCK>(total, total, c1s, c2s, as, nb_off, nb, &fb, err, tally)
            : decimate_round_passes<BLOCK>(total, total, c1g, c2g, alive, nb_off, nb, &fb, err, tally);
        if (tid == 0) {
            s_alive = left;
            s_fallback = fb;
        }
        __syncthreads();
        if (in_smem)
            for (int i = tid; i < total; i += BLOCK) alive[i] = as[i];
        __syncthreads();
        if (!s_fallback) return;
    }
    if (in_smem) {
        // Candidate bitmap: bit i set <=> point i is alive and removable now.
        // The in-order scan then jumps from candidate to candidate; a removal
        // re-evaluates exactly the neighbours whose counts it changed, so the
        // bitmap stays exact and the scan visits what the sequential list
        // walk of decimate.hpp would remove, in the same order.
        const int nwords = (total + 31) >> 5;
        for (int i0 = 0; i0 < nwords * 32; i0 += BLOCK) {
            const int i = i0 + tid;
            const bool q = (i < total) && as[i] && (c1s[i] >= 4 || c2s[i] < 3);
            const unsigned bal = __ballot_sync(FULL, q);
            if (lane == 0 && (i >> 5) < nwords) cand[i >> 5] = bal;
        }
        __syncthreads();
        // A removal decrements the counts of its listed neighbours (distinct
        // points, one thread each) and re-evaluates their candidate bits.
        auto update = [&](int t) {
            const int e = nb[t];
            const int q = e & 0x7fffffff;
            const int a = (c1s[q] -= (e < 0) ? 1 : 0);
            const int b = (c2s[q] -= 1);
            const uint32_t bit = 1u << (q & 31);
            if (as[q] && (a >= 4 || b < 3)) atomicOr(&cand[q >> 5], bit);
            else atomicAnd(&cand[q >> 5], ~bit);
        };
        // Warp 0 drives the scan; a list longer than DEC_WIDE_LIST is
        // processed by the whole CTA: the other warps wait on named barrier 1
        // for a command (list range, or -1 = done) and report completion on
        // named barrier 2.
        constexpr int DEC_WIDE_LIST = 96;
        __shared__ int s_cmd[2];
        if (warp == 0) {
            // first candidate >= pos, or -1
            auto next_cand = [&](int pos) -> int {
                int wi = pos >> 5;
                if (wi >= nwords) return -1;
                const uint32_t first = cand[wi] & (0xffffffffu << (pos & 31));
                if (first) return (wi << 5) + __ffs(first) - 1;
                for (int w0 = wi + 1; w0 < nwords; w0 += 32) {
                    const int w = w0 + lane;
                    const uint32_t word = (w < nwords) ? cand[w] : 0u;
                    const unsigned bal = __ballot_sync(FULL, word != 0u);
                    if (bal) {
                        const int src = __ffs(bal) - 1;
                        const uint32_t wb = __shfl_sync(FULL, word, src);
                        return ((w0 + src) << 5) + __ffs(wb) - 1;
                    }
                }
                return -1;
            };
            int cnt = s_alive, left = -1, guard = 0;
            bool stop = false;
            while (left != cnt && cnt > 3 && !stop) {
                if (++guard > total + 2) { if (lane == 0) atomicOr(err, ERRB_DEC_CAP); break; }
                left = cnt;
                int pos = 0;
                for (;;) {
                    const int j = next_cand(pos);
                    if (j < 0) break;
                    if (nocopy && cnt - 1 < 3) { stop = true; break; }
                    if (lane == 0) {
                        as[j] = 0;
                        alive[j] = 0;
                        atomicAnd(&cand[j >> 5], ~(1u << (j & 31)));
                    }
                    --cnt;
                    const int e0 = nb_off[j], e1 = nb_off[j + 1];
                    if (BLOCK > 32 && e1 - e0 > DEC_WIDE_LIST) {
                        if (lane == 0) { s_cmd[0] = e0; s_cmd[1] = e1; }
                        named_bar_sync(1, BLOCK);
                        for (int t = e0 + lane; t < e1; t += BLOCK) update(t);
                        named_bar_sync(2, BLOCK);
                    } else {
                        for (int t = e0 + lane; t < e1; t += 32) update(t);
                        __syncwarp();
                    }
                    if (!nocopy && cnt < 3) break;
                    pos = j + 1;
                }
                if (!nocopy && cnt < 3) break;
            }
            if (BLOCK > 32) {
                if (lane == 0) s_cmd[0] = -1;
                named_bar_sync(1, BLOCK);
            }
        } else {
            for (;;) {
                named_bar_sync(1, BLOCK);
                const int e0 = s_cmd[0];
                if (e0 < 0) break;
                const int e1 = s_cmd[1];
                for (int t = e0 + tid; t < e1; t += BLOCK) update(t);
                named_bar_sync(2, BLOCK);
            }
        }
        __syncthreads();
        return;
    }
    // sequential in-order scan (warp 0), as decimate_scan
    if (warp == 0) {
        auto get_alive = [&](int w) -> bool { return in_smem ? as[w] != 0 : alive[w] != 0; };
        auto removable = [&](int w) -> bool {
            const int a = in_smem ? c1s[w] : c1g[w];
            const int b = in_smem ? c2s[w] : c2g[w];
            return a >= 4 || b < 3;
        };
        int cnt = s_alive, left = -1, guard = 0;
        bool stop = false;
        while (left != cnt && cnt > 3 && !stop) {
            if (++guard > total + 2) { if (lane == 0) atomicOr(err, ERRB_DEC_CAP); break; }
            left = cnt;
            int i = 0;
            while (i < total) {
                const int w = i + lane;
                const bool pred = (w < total) && get_alive(w) && removable(w);
                const unsigned bal = __ballot_sync(FULL, pred);
                if (bal == 0) { i += 32; continue; }
                const int j = i + __ffs(bal) - 1;
                if (nocopy && cnt - 1 < 3) { stop = true; break; }
                if (lane == 0) {
                    if (in_smem) as[j] = 0;
                    alive[j] = 0;
                }
                --cnt;
                const int e0 = nb_off[j], e1 = nb_off[j + 1];
                for (int t = e0 + lane; t < e1; t += 32) {  // distinct neighbours per lane
                    const int e = nb[t];
                    const int q = e & 0x7fffffff;
                    if (in_smem) {
                        c2s[q] -= 1;
                        if (e < 0) c1s[q] -= 1;
                    } else {
                        c2g[q] -= 1;
                        if (e < 0) c1g[q] -= 1;
                    }
                }
                __syncwarp();
                if (!nocopy && cnt < 3) break;
                i = j + 1;
            }
            if (!nocopy && cnt < 3) break;
        }
    }
    __syncthreads();
}

}  // namespace
}  // namespace rdb
