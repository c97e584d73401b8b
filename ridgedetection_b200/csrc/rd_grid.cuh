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

}  // namespace
}  // namespace rdb
