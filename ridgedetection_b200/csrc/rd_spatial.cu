// rd_spatial.cu -- spatial order of the evolve points for the culled
// assignment (k_assign_cull in rd_kernels.cu).
//
// The brute-force assignment of rd/cpu/brute_force/evolve.hpp:43-66 keeps a
// point's nearest chosen point only when it lies within r1.  A group of points
// that are close together in space therefore needs only the chosen points
// within r1 of the group's bounding box.  This file builds, once per run (the
// evolve points never move), a copy of every cloud's points in a spatial
// order -- cells of edge r1/4, Morton order of the cells, the packed slot
// order inside a cell.  The copy pads DIM 3 to four floats per point, so that
// a point is one 16-byte load.
#include "rd_engine.cuh"

#include <cub/cub.cuh>

#include <algorithm>
#include <cmath>
#include <cstdint>

namespace rdb {
namespace {

// x's low 16 bits moved to the even bit positions
__device__ __forceinline__ uint32_t spread_by_1(uint32_t x)
{
    x &= 0xffffu;
    x = (x | (x << 8)) & 0x00ff00ffu;
    x = (x | (x << 4)) & 0x0f0f0f0fu;
    x = (x | (x << 2)) & 0x33333333u;
    x = (x | (x << 1)) & 0x55555555u;
    return x;
}

// x's low 10 bits moved to every third bit position
__device__ __forceinline__ uint32_t spread_by_2(uint32_t x)
{
    x &= 0x3ffu;
    x = (x | (x << 16)) & 0x030000ffu;
    x = (x | (x << 8)) & 0x0300f00fu;
    x = (x | (x << 4)) & 0x030c30c3u;
    x = (x | (x << 2)) & 0x09249249u;
    return x;
}

template <int DIM>
__device__ __forceinline__ uint32_t morton_code(const float* p, float inv)
{
    // the order only affects how tight the culling boxes are: one dimension
    // sorts by its cell, four and more interleave the first three
    if constexpr (DIM == 1) {
        return spatial_cell(p[0], inv);
    } else if constexpr (DIM == 2) {
        return spread_by_1(spatial_cell(p[0], inv)) | (spread_by_1(spatial_cell(p[1], inv)) << 1);
    } else {
        return spread_by_2(spatial_cell(p[0], inv)) | (spread_by_2(spatial_cell(p[1], inv)) << 1) |
               (spread_by_2(spatial_cell(p[2], inv)) << 2);
    }
}

// chunk lc of cloud cd covers positions [lo, hi) of the cloud
__device__ __forceinline__ void chunk_range(const CloudDesc& cd, int lc, int& lo, int& hi)
{
    lo = (int)(((int64_t)lc * cd.n_all) / cd.n_chunks);
    hi = (int)(((int64_t)(lc + 1) * cd.n_all) / cd.n_chunks);
}

// sort keys: (cloud << 32) | Morton code; values: packed slot
template <int DIM>
__global__ void __launch_bounds__(256) k_morton(EngineView v, uint64_t* key, int32_t* val)
{
    for (int ch = blockIdx.x; ch < v.n_chunks; ch += gridDim.x) {
        const int c = v.chunk_cloud[ch];
        const CloudDesc cd = v.cl[c];
        int lo, hi;
        chunk_range(cd, (int)(ch - cd.chunk_begin), lo, hi);
        const float inv = spatial_cell_inv(cd.r1);
        for (int i = lo + threadIdx.x; i < hi; i += blockDim.x) {
            const int64_t s = cd.p_off + i;
            float p[DIM];
#pragma unroll
            for (int d = 0; d < DIM; ++d) p[d] = v.P[s * DIM + d];
            key[s] = ((uint64_t)(uint32_t)c << 32) | morton_code<DIM>(p, inv);
            val[s] = (int32_t)s;
        }
    }
}

// Ps, sorder, and (second half of sorder) each position's histogram row: the
// chunk of its slot inside its cloud, from the sorted keys' cloud field
template <int DIM>
__global__ void __launch_bounds__(256) k_gather_spatial(EngineView v, int64_t n, const int32_t* val,
                                                        const uint64_t* key, float* Ps,
                                                        int32_t* sorder)
{
    constexpr int DP = PadDim<DIM>::v;
    for (int64_t pos = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; pos < n;
         pos += (int64_t)gridDim.x * blockDim.x) {
        const int32_t s = val[pos];
        const CloudDesc cd = v.cl[(int)(key[pos] >> 32)];
        sorder[n + pos] = slot_chunk((int)(s - cd.p_off), cd.n_all, cd.n_chunks,
                                     (float)cd.n_chunks / (float)cd.n_all);
#pragma unroll
        for (int d = 0; d < DIM; ++d) Ps[pos * DP + d] = v.P[(int64_t)s * DIM + d];
#pragma unroll
        for (int d = DIM; d < DP; ++d) Ps[pos * DP + d] = 0.0f;
        sorder[pos] = s;
    }
}

size_t sort_temp_bytes(int64_t n)
{
    size_t bytes = 0;
    cub::DoubleBuffer<uint64_t> k(nullptr, nullptr);
    cub::DoubleBuffer<int32_t> v(nullptr, nullptr);
    cub::DeviceRadixSort::SortPairs(nullptr, bytes, k, v, (int)n, 0, 64);
    return bytes;
}

size_t align256(size_t x) { return (x + 255) / 256 * 256; }

template <int DIM>
cudaError_t spatial_prep_dim(const EngineView& v, int64_t n, void* scratch, size_t scratch_bytes,
                             float* Ps, int32_t* sorder, cudaStream_t st)
{
    if (n <= 0 || v.n_chunks <= 0) return cudaSuccess;
    unsigned char* p = static_cast<unsigned char*>(scratch);
    uint64_t* k0 = reinterpret_cast<uint64_t*>(p);
    uint64_t* k1 = reinterpret_cast<uint64_t*>(p + align256(8 * (size_t)n));
    int32_t* v0 = reinterpret_cast<int32_t*>(p + 2 * align256(8 * (size_t)n));
    int32_t* v1 = reinterpret_cast<int32_t*>(p + 2 * align256(8 * (size_t)n) + align256(4 * (size_t)n));
    unsigned char* tmp = p + 2 * align256(8 * (size_t)n) + 2 * align256(4 * (size_t)n);
    const size_t used = (size_t)(tmp - p);
    if (scratch_bytes < used) return cudaErrorInvalidValue;
    size_t tmp_bytes = scratch_bytes - used;
    const int sms = v.n_sms > 0 ? v.n_sms : 148;
    const int cgrid = std::max(1, std::min(v.n_chunks, sms * 8));
    k_morton<DIM><<<cgrid, 256, 0, st>>>(v, k0, v0);
    int end_bit = 32;
    while (end_bit < 64 && (int64_t(1) << (end_bit - 32)) < v.n_clouds) ++end_bit;
    cub::DoubleBuffer<uint64_t> kb(k0, k1);
    cub::DoubleBuffer<int32_t> vb(v0, v1);
    cudaError_t e = cub::DeviceRadixSort::SortPairs(tmp, tmp_bytes, kb, vb, (int)n, 0, end_bit, st);
    if (e != cudaSuccess) return e;
    const int ggrid = (int)std::max<int64_t>(1, std::min<int64_t>((n + 255) / 256, (int64_t)sms * 16));
    k_gather_spatial<DIM><<<ggrid, 256, 0, st>>>(v, n, vb.Current(), kb.Current(), Ps, sorder);
    return cudaGetLastError();
}

}  // namespace

size_t spatial_prep_scratch_bytes(int64_t n)
{
    if (n <= 0) return 256;
    return 2 * align256(8 * (size_t)n) + 2 * align256(4 * (size_t)n) + align256(sort_temp_bytes(n));
}

cudaError_t launch_spatial_prep(int dim, const EngineView& v, int64_t n, void* scratch,
                                size_t scratch_bytes, float* Ps, int32_t* sorder, cudaStream_t st)
{
    switch (dim) {
        case 1: return spatial_prep_dim<1>(v, n, scratch, scratch_bytes, Ps, sorder, st);
        case 2: return spatial_prep_dim<2>(v, n, scratch, scratch_bytes, Ps, sorder, st);
        case 3: return spatial_prep_dim<3>(v, n, scratch, scratch_bytes, Ps, sorder, st);
        case 4: return spatial_prep_dim<4>(v, n, scratch, scratch_bytes, Ps, sorder, st);
        default: return cudaErrorInvalidValue;
    }
}

}  // namespace rdb
