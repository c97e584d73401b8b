// rd_adjoint.cu -- reverse pass of `iters` evolve passes (no reference
// counterpart; the reference is forward-only).
//
// Forward, on the engine with the movement test switched off: A^t is the exact
// assignment of the cloud to S^{t-1} (the brute-force assign kernel), and
// S^t_k = (FP32 sum of A^t_k in index order) / |A^t_k| for |A^t_k| > 0, else
// S^{t-1}_k.  Loss L = sum_k <W_k, S^iters_k>.
// Reverse, assignments frozen, FP64: g = W; for t = iters..1 every member i of
// a non-empty cluster k gets g_k / |A^t_k| added to dL/dP_i and g_k is reset;
// empty clusters carry g_k to S^{t-1}.  What is left of g is dL/dS^0.
// Memory: all assignments are kept (iters x N ints) when checkpoint_every = 0;
// otherwise S is checkpointed every `checkpoint_every` passes and the
// assignments of one segment at a time are recomputed during the reverse pass.
#include "rd_adjoint.hpp"

#include <algorithm>
#include <cstring>

namespace rdb {

namespace {

template <int DIM>
__global__ void k_adj_members(const int32_t* __restrict__ keys, const int32_t* __restrict__ cnt,
                              const double* __restrict__ g, int64_t n, double* __restrict__ gP)
{
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        const int k = keys[i];
        if (k < 0) continue;
        const double inv = 1.0 / (double)cnt[k];
#pragma unroll
        for (int d = 0; d < DIM; ++d) gP[i * DIM + d] += g[(int64_t)k * DIM + d] * inv;
    }
}

template <int DIM>
__global__ void k_adj_carry(const int32_t* __restrict__ cnt, int64_t ns, double* __restrict__ g)
{
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < ns;
         k += (int64_t)gridDim.x * blockDim.x)
        if (cnt[k] > 0)
#pragma unroll
            for (int d = 0; d < DIM; ++d) g[k * DIM + d] = 0.0;
}

int grid_for(int64_t n) { return (int)std::max<int64_t>(1, std::min<int64_t>((n + 255) / 256, 148 * 16)); }

}  // namespace

int AdjointRunner::fail(const char* what, cudaError_t e)
{
    last_error = std::string(what) + ": " + cudaGetErrorString(e);
    return 2;
}

#define AK(call)                                      \
    do {                                              \
        cudaError_t e_ = (call);                      \
        if (e_ != cudaSuccess) return fail(#call, e_); \
    } while (0)

int AdjointRunner::run(int dim, const float* d_P, int64_t np, const float* d_S0, int64_t ns,
                       float r1, int iters, int ckpt, const double* d_W, float* d_S_final,
                       double* d_gP, double* d_gS0, cudaStream_t st)
{
    if (!dim_supported(dim)) { last_error = "dim must be 1 to 4"; return 6; }
    if (np < 1 || ns < 1 || ns > np || iters < 0 || ckpt < 0) { last_error = "bad sizes"; return 1; }
    CloudDesc cd;
    std::memset(&cd, 0, sizeof(cd));
    cd.n_all = (int32_t)np;
    cd.n_own = (int32_t)np;
    cd.r1 = r1;
    cd.r2 = r1;
    GroupDesc gd;
    std::memset(&gd, 0, sizeof(gd));
    gd.n_clouds = 1;
    if (int rc = eng_.setup(dim, {cd}, {gd}, np)) { last_error = eng_.last_error; return rc; }
    AK(cudaMemcpyAsync(eng_.points(), d_P, sizeof(float) * np * dim, cudaMemcpyDeviceToDevice, st));
    AK(cudaMemcpyAsync(eng_.chosen_mut(), d_S0, sizeof(float) * ns * dim, cudaMemcpyDeviceToDevice, st));
    eng_.given_ns.assign(1, (int32_t)ns);
    if (int rc = eng_.adjoint_setup(st)) { last_error = eng_.last_error; return rc; }
    const int seg = ckpt > 0 ? ckpt : std::max(iters, 1);
    const int nseg = (iters + seg - 1) / seg;
    AK(bKeys_.ensure(sizeof(int32_t) * (size_t)np * seg + 16));
    AK(bCnt_.ensure(sizeof(int32_t) * (size_t)ns * seg + 16));
    AK(bCkpt_.ensure(sizeof(float) * (size_t)ns * dim * (nseg + 1) + 16));
    AK(bG_.ensure(sizeof(double) * (size_t)ns * dim + 16));
    float* S = eng_.chosen_mut();
    const size_t sbytes = sizeof(float) * ns * dim;
    auto keep = [&](int slot) -> int {
        AK(cudaMemcpyAsync(bKeys_.as<int32_t>() + (size_t)slot * np, eng_.keys(),
                           sizeof(int32_t) * np, cudaMemcpyDeviceToDevice, st));
        AK(cudaMemcpyAsync(bCnt_.as<int32_t>() + (size_t)slot * ns, eng_.counts(),
                           sizeof(int32_t) * ns, cudaMemcpyDeviceToDevice, st));
        return 0;
    };
    // forward, checkpointing S at the start of every segment
    for (int t = 0; t < iters; ++t) {
        if (t % seg == 0)
            AK(cudaMemcpyAsync(bCkpt_.as<float>() + (size_t)(t / seg) * ns * dim, S, sbytes,
                               cudaMemcpyDeviceToDevice, st));
        if (int rc = eng_.adjoint_step(st)) { last_error = eng_.last_error; return rc; }
        if (nseg == 1)
            if (int rc = keep(t)) return rc;
    }
    if (d_S_final) AK(cudaMemcpyAsync(d_S_final, S, sbytes, cudaMemcpyDeviceToDevice, st));
    // reverse
    AK(cudaMemcpyAsync(bG_.p, d_W, sizeof(double) * ns * dim, cudaMemcpyDeviceToDevice, st));
    AK(cudaMemsetAsync(d_gP, 0, sizeof(double) * np * dim, st));
    for (int s = nseg - 1; s >= 0; --s) {
        const int t0 = s * seg, t1 = std::min(iters, t0 + seg);
        if (nseg > 1) {  // recompute the segment's assignments from its checkpoint
            AK(cudaMemcpyAsync(S, bCkpt_.as<float>() + (size_t)s * ns * dim, sbytes,
                               cudaMemcpyDeviceToDevice, st));
            for (int t = t0; t < t1; ++t) {
                if (int rc = eng_.adjoint_step(st)) { last_error = eng_.last_error; return rc; }
                if (int rc = keep(t - t0)) return rc;
            }
        }
        for (int t = t1 - 1; t >= t0; --t) {
            const int slot = (nseg > 1) ? t - t0 : t;
            const int32_t* kt = bKeys_.as<int32_t>() + (size_t)slot * np;
            const int32_t* ct = bCnt_.as<int32_t>() + (size_t)slot * ns;
            AK(with_dim(dim, [&](auto D) {
                constexpr int DIM = decltype(D)::value;
                k_adj_members<DIM><<<grid_for(np), 256, 0, st>>>(kt, ct, bG_.as<double>(), np, d_gP);
                k_adj_carry<DIM><<<grid_for(ns), 256, 0, st>>>(ct, ns, bG_.as<double>());
                return cudaGetLastError();
            }));
        }
    }
    if (d_gS0) AK(cudaMemcpyAsync(d_gS0, bG_.p, sizeof(double) * ns * dim, cudaMemcpyDeviceToDevice, st));
    AK(cudaStreamSynchronize(st));
    return 0;
}

}  // namespace rdb
