// rd_quality.cu -- quality metrics of a ridge on the device
// (rd/utils/assessment_quality.hpp), with the reference's float arithmetic:
//   distance(p, B)  = sqrt(min over B of the squared distance p - b)
//   Hausdorff(T, I) = max(max over T of distance(t, I), max over I of distance(i, T))
//   stats(S, I)     = min, max, median (sorted[n/2]) and mean (float sum in
//                     sorted order / n) of distance(s, I)
//   segment(T)      = max over T of sqrt(sum over d >= 1 of t_d^2)
// The min-distance search is all pairs, one thread per four points against
// shared-memory tiles of the other set; the mean's ordered sum uses the exact
// parallel fold (rd_fold.cuh), so it equals the sequential float sum.
#include "rd_engine.cuh"
#include "rd_fold.cuh"

#include <cfloat>
#include <cub/cub.cuh>
#include <cuda_runtime.h>

namespace rdb {
namespace {

constexpr int Q_BLOCK = 256, Q_ITEMS = 4, Q_TILE = 1024;

template <int DIM>
__global__ void __launch_bounds__(Q_BLOCK) k_min_dist(const float* __restrict__ A, int na,
                                                      const float* __restrict__ B, int nb,
                                                      float* __restrict__ out)
{
    __shared__ float sB[Q_TILE * DIM];
    const int tid = threadIdx.x;
    const int i0 = blockIdx.x * Q_BLOCK * Q_ITEMS + tid;
    float p[Q_ITEMS][DIM], best[Q_ITEMS];
#pragma unroll
    for (int j = 0; j < Q_ITEMS; ++j) {
        const int i = i0 + j * Q_BLOCK;
#pragma unroll
        for (int d = 0; d < DIM; ++d) p[j][d] = (i < na) ? A[(int64_t)i * DIM + d] : 0.0f;
        best[j] = FLT_MAX;
    }
    for (int t0 = 0; t0 < nb; t0 += Q_TILE) {
        const int tl = min(Q_TILE, nb - t0);
        __syncthreads();
        for (int e = tid; e < tl * DIM; e += Q_BLOCK) sB[e] = B[(int64_t)t0 * DIM + e];
        __syncthreads();
        for (int k = 0; k < tl; ++k) {
            float s[DIM];
#pragma unroll
            for (int d = 0; d < DIM; ++d) s[d] = sB[k * DIM + d];
#pragma unroll
            for (int j = 0; j < Q_ITEMS; ++j) {
                const float dd = sqdist_exact<DIM>(p[j], s);
                if (dd < best[j]) best[j] = dd;
            }
        }
    }
#pragma unroll
    for (int j = 0; j < Q_ITEMS; ++j) {
        const int i = i0 + j * Q_BLOCK;
        if (i < na) out[i] = sqrtf(best[j]);
    }
}

template <int DIM>
__global__ void __launch_bounds__(256) k_axis_dist(const float* __restrict__ T, int n,
                                                  float* __restrict__ out)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float s = 0.0f;
#pragma unroll
    for (int k = 1; k < DIM; ++k) {
        const float x = T[(int64_t)i * DIM + k];
        s = __fadd_rn(s, __fmul_rn(x, x));
    }
    out[i] = (s > 0.0f) ? sqrtf(s) : 0.0f;
}

// largest value of a[0..na) and b[0..nb) (one CTA)
__global__ void __launch_bounds__(1024) k_max2(const float* a, int na, const float* b, int nb,
                                               float* out)
{
    __shared__ float s_w[32];
    float m = -FLT_MAX;
    for (int i = threadIdx.x; i < na; i += 1024) m = fmaxf(m, a[i]);
    for (int i = threadIdx.x; i < nb; i += 1024) m = fmaxf(m, b[i]);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0) s_w[threadIdx.x >> 5] = m;
    __syncthreads();
    if (threadIdx.x < 32) {
        m = s_w[threadIdx.x];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
        if (threadIdx.x == 0) *out = m;
    }
}

__global__ void k_iota(int32_t* idx, int n)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) idx[i] = i;
}

// {median, mean, min, max} of the sorted distances (one CTA of 256 threads)
__global__ void __launch_bounds__(256) k_stats(const float* sorted, const int32_t* iota, int n,
                                              float* out)
{
    __shared__ FoldCtaSmem<8, 1> sm;
    fold_members_cta<8, 1>(iota, n, sorted, sm);
    if (threadIdx.x == 0) {
        out[0] = sorted[n / 2];
        out[1] = __fdiv_rn(sm.s[0], (float)n);
        out[2] = sorted[0];
        out[3] = sorted[n - 1];
    }
}

inline int q_grid(int n) { return (n + Q_BLOCK * Q_ITEMS - 1) / (Q_BLOCK * Q_ITEMS); }

}  // namespace

cudaError_t launch_min_dist(int dim, const float* A, int na, const float* B, int nb, float* out,
                            cudaStream_t st)
{
    if (na <= 0) return cudaSuccess;
    return with_dim(dim, [&](auto D) {
        k_min_dist<decltype(D)::value><<<q_grid(na), Q_BLOCK, 0, st>>>(A, na, B, nb, out);
        return cudaGetLastError();
    });
}

cudaError_t launch_axis_dist(int dim, const float* T, int n, float* out, cudaStream_t st)
{
    if (n <= 0) return cudaSuccess;
    return with_dim(dim, [&](auto D) {
        k_axis_dist<decltype(D)::value><<<(n + 255) / 256, 256, 0, st>>>(T, n, out);
        return cudaGetLastError();
    });
}

cudaError_t launch_max2(const float* a, int na, const float* b, int nb, float* out, cudaStream_t st)
{
    k_max2<<<1, 1024, 0, st>>>(a, na, b, nb, out);
    return cudaGetLastError();
}

// sorts d (n floats, all >= 0) through the scratch and writes {median, mean,
// min, max} to out (device); scratch: 2n floats + n ints + cub storage
cudaError_t launch_dist_stats(float* d, int n, float* sorted, int32_t* iota, void* temp,
                              size_t temp_bytes, float* out, cudaStream_t st)
{
    cudaError_t e = cub::DeviceRadixSort::SortKeys(temp, temp_bytes, d, sorted, n, 0, 32, st);
    if (e != cudaSuccess) return e;
    k_iota<<<(n + 255) / 256, 256, 0, st>>>(iota, n);
    k_stats<<<1, 256, 0, st>>>(sorted, iota, n, out);
    return cudaGetLastError();
}

size_t dist_stats_temp_bytes(int n)
{
    size_t bytes = 0;
    cub::DeviceRadixSort::SortKeys(nullptr, bytes, (float*)nullptr, (float*)nullptr, n, 0, 32);
    return bytes;
}

}  // namespace rdb
