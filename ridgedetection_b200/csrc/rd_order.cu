// rd_order.cu -- ordering of a ridge into chains (rd/cpu/brute_force/order.hpp:45-141,
// with the condition the brute-force class passes, ridge_detection.inl:148-168).
//
// Every remaining point, in index order, seeds a chain.  The chain then takes,
// again and again, the first later remaining point (lowest index) that is
// within r2 of its front -- tested first -- or of its back, until none is
// left.  Each step depends on the last, but "the first remaining point within
// r2 of either end" is a min-index search over all later points, which one
// CTA does in parallel: every thread scans its stride of candidates up to its
// first hit, then a block-wide min picks the winner.  The chain grows in a
// deque (front and back indices around the middle of a 2*ns+1 buffer) and is
// written out front to back.
#include "rd_engine.cuh"

#include <climits>
#include <cuda_runtime.h>

namespace rdb {
namespace {

constexpr int ORDER_BLOCK = 1024;

template <int DIM>
__global__ void __launch_bounds__(ORDER_BLOCK)
    k_order_chains(const float* __restrict__ S, int ns, float rsq, unsigned char* alive,
                   int32_t* deq, int32_t* order, int32_t* chain_start, int32_t* n_chains)
{
    __shared__ int s_min[ORDER_BLOCK / 32];
    __shared__ int s_hit, s_head, s_tail;
    __shared__ float s_f[DIM], s_b[DIM];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    for (int i = tid; i < ns; i += ORDER_BLOCK) alive[i] = 1;
    __syncthreads();
    int out = 0, nch = 0;  // the same in every thread
    for (int p = 0; p < ns; ++p) {
        if (!alive[p]) continue;  // written by thread 0 before a barrier: uniform
        __syncthreads();
        if (tid == 0) {
            alive[p] = 0;
            deq[ns] = p;
            s_head = ns;
            s_tail = ns;
#pragma unroll
            for (int d = 0; d < DIM; ++d) s_f[d] = s_b[d] = S[(int64_t)p * DIM + d];
        }
        __syncthreads();
        for (;;) {
            float f[DIM], b[DIM];
#pragma unroll
            for (int d = 0; d < DIM; ++d) {
                f[d] = s_f[d];
                b[d] = s_b[d];
            }
            int best = INT_MAX;
            for (int j = p + 1 + tid; j < ns; j += ORDER_BLOCK) {
                if (!alive[j]) continue;
                float q[DIM];
#pragma unroll
                for (int d = 0; d < DIM; ++d) q[d] = S[(int64_t)j * DIM + d];
                if (sqdist_exact<DIM>(q, f) <= rsq || sqdist_exact<DIM>(q, b) <= rsq) {
                    best = j;
                    break;
                }
            }
            const int m = __reduce_min_sync(0xffffffffu, best);
            if (lane == 0) s_min[warp] = m;
            __syncthreads();
            if (warp == 0) {
                const int v = __reduce_min_sync(0xffffffffu, (lane < ORDER_BLOCK / 32) ? s_min[lane] : INT_MAX);
                if (lane == 0) s_hit = v;
            }
            __syncthreads();
            const int hit = s_hit;
            if (hit == INT_MAX) break;
            if (tid == 0) {
                alive[hit] = 0;
                float q[DIM];
#pragma unroll
                for (int d = 0; d < DIM; ++d) q[d] = S[(int64_t)hit * DIM + d];
                if (sqdist_exact<DIM>(q, f) <= rsq) {
                    deq[--s_head] = hit;
#pragma unroll
                    for (int d = 0; d < DIM; ++d) s_f[d] = q[d];
                } else {
                    deq[++s_tail] = hit;
#pragma unroll
                    for (int d = 0; d < DIM; ++d) s_b[d] = q[d];
                }
            }
            __syncthreads();
        }
        const int head = s_head, tail = s_tail;
        for (int k = head + tid; k <= tail; k += ORDER_BLOCK) order[out + (k - head)] = deq[k];
        if (tid == 0) chain_start[nch] = out;
        out += tail - head + 1;
        ++nch;
        __syncthreads();  // the deque is reused by the next chain
    }
    if (tid == 0) {
        chain_start[nch] = out;
        *n_chains = nch;
    }
}

}  // namespace

cudaError_t launch_order_chains(int dim, const float* S, int ns, float rsq, unsigned char* alive,
                                int32_t* deq, int32_t* order, int32_t* chain_start,
                                int32_t* n_chains, cudaStream_t st)
{
    return with_dim(dim, [&](auto D) {
        k_order_chains<decltype(D)::value><<<1, ORDER_BLOCK, 0, st>>>(S, ns, rsq, alive, deq, order,
                                                                     chain_start, n_chains);
        return cudaGetLastError();
    });
}

}  // namespace rdb
