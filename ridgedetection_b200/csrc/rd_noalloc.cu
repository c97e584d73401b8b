// rd_noalloc.cu -- decimation that allocates no device memory.
//
// Some callers cannot call cudaMalloc: real-time or embedded hosts that
// forbid device allocation once they have started (an allocation can block
// for a long time or fail under memory pressure), and plugins whose device
// memory is owned by a framework that does not hand out a workspace.
// rd_decimate_noalloc serves them: its scratch lives in one file-scope
// __device__ array of fixed size, so a call only launches kernels.
//
// The array is RD_DECIMATE_NOALLOC_SCRATCH_BYTES (1.5 MiB) on every GPU
// that loads the library, held until the process exits.  Every call uses the
// same array: two calls whose kernels overlap on the GPU (different streams,
// or different host threads) race on it.  Each call clears what must start
// at zero (bucket counts, error flag) and overwrites the rest before reading.
#include "../../include/rd_c_api.h"
#include "rd_grid.cuh"

#include <cuda.h>

#include <mutex>
#include <string>

namespace rdb {

rd_status report_error(rd_status s, const char* msg);  // per-thread message (rd_capi.cu)

namespace {

constexpr int NA_MAX = RD_DECIMATE_NOALLOC_MAX_POINTS;
constexpr int NA_HBITS = 15;                    // 2^15 buckets >= NA_MAX
constexpr int64_t NA_INTS = (int64_t)NA_MAX * (3 + 3 + 4) + (1 << NA_HBITS) + 1 + 16;
static_assert(NA_INTS * 4 <= RD_DECIMATE_NOALLOC_SCRATCH_BYTES, "scratch size");

// The scratch.  In host code this name is only a host-side handle: its device
// address comes from cudaGetSymbolAddress (once per device, below).
static __device__ __align__(256) int32_t g_noalloc_scratch[RD_DECIMATE_NOALLOC_SCRATCH_BYTES / 4];

template <int DIM, int BLOCK>
__global__ void __launch_bounds__(BLOCK) k_decimate_noalloc(float* S, int ns, float r2,
                                                            int32_t* ns_out, int32_t* scratch)
{
    float* X = reinterpret_cast<float*>(scratch);          // NA_MAX * 3
    int32_t* cell = scratch + NA_MAX * 3;                   // NA_MAX * 3
    int32_t* alive = cell + NA_MAX * 3;
    int32_t* c1 = alive + NA_MAX;
    int32_t* c2 = c1 + NA_MAX;
    int32_t* items = c2 + NA_MAX;
    int32_t* bstart = items + NA_MAX;                       // 2^NA_HBITS + 1
    int32_t* err = bstart + (1 << NA_HBITS) + 1;
    __shared__ int s_off[BLOCK / 32];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    for (int e = tid; e < ns * DIM; e += BLOCK) X[e] = S[e];
    if (tid == 0) *err = 0;
    int hbits = 6;
    while ((1 << hbits) < ns && hbits < NA_HBITS) ++hbits;
    decimate_scan<DIM, BLOCK>(X, ns, r2, 0, cell, alive, c1, c2, items, bstart,
                              (1u << hbits) - 1, err);
    // survivors back into S, in order
    int kept = 0;
    for (int k0 = 0; k0 < ns; k0 += BLOCK) {
        const int k = k0 + tid;
        const bool a = (k < ns) && alive[k];
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
            for (int d = 0; d < DIM; ++d) S[(int64_t)pos * DIM + d] = X[(int64_t)k * DIM + d];
        }
        kept += tot;
        __syncthreads();
    }
    if (tid == 0) *ns_out = (*err) ? -1 : kept;
}

constexpr int MAX_DEVICES = 64;
std::mutex g_mu;
struct ScratchAddr {
    unsigned long long ctx_id;   // context the address belongs to (0 = not looked up)
    int32_t* ptr;
};
ScratchAddr g_dev_addr[MAX_DEVICES] = {};

// Identifier of the calling thread's current context (cuCtxGetId, resolved
// through the runtime so the library needs no libcuda link); 0 when it
// cannot be had, in which case the address is looked up on every call.
unsigned long long current_context_id()
{
    using GetCurrent = CUresult (*)(CUcontext*);
    using GetId = CUresult (*)(CUcontext, unsigned long long*);
    static GetCurrent get_current = nullptr;
    static GetId get_id = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void* f = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            get_current = reinterpret_cast<GetCurrent>(f);
        f = nullptr;
        if (cudaGetDriverEntryPoint("cuCtxGetId", &f, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            get_id = reinterpret_cast<GetId>(f);
    });
    CUcontext ctx = nullptr;
    unsigned long long id = 0;
    if (!get_current || !get_id || get_current(&ctx) != CUDA_SUCCESS || !ctx) return 0;
    if (get_id(ctx, &id) != CUDA_SUCCESS) return 0;
    return id;
}

// Device address of the scratch on the current device, looked up with that
// device current the first time it is used in a context.  A device reset
// destroys the context and may reload the module elsewhere, so the address is
// keyed on the context and looked up again in a new one.
cudaError_t scratch_on_current_device(int32_t** out)
{
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= MAX_DEVICES) return cudaErrorInvalidDevice;
    unsigned long long ctx = current_context_id();
    std::lock_guard<std::mutex> lk(g_mu);
    if (ctx == 0 || g_dev_addr[dev].ctx_id != ctx || !g_dev_addr[dev].ptr) {
        void* p = nullptr;
        e = cudaGetSymbolAddress(&p, g_noalloc_scratch);   // creates the context if needed
        if (e != cudaSuccess) return e;
        if (ctx == 0) ctx = current_context_id();
        g_dev_addr[dev].ctx_id = ctx;
        g_dev_addr[dev].ptr = static_cast<int32_t*>(p);
    }
    *out = g_dev_addr[dev].ptr;
    return cudaSuccess;
}

}  // namespace

int decimate_noalloc(int dim, float* d_S, int64_t ns, float r2, int32_t* d_ns_out,
                     cudaStream_t st)
{
    if (dim != 2 && dim != 3) return report_error(RD_ERR_UNSUPPORTED, "dim must be 2 or 3");
    if (!d_S || !d_ns_out || ns < 0 || !(r2 > 0.0f))
        return report_error(RD_ERR_ARG, "null pointer, negative count or r2 <= 0");
    if (ns > NA_MAX) {
        const std::string msg = "rd_decimate_noalloc: " + std::to_string(ns) +
                                " points exceed the fixed scratch limit of " + std::to_string(NA_MAX) +
                                " (RD_DECIMATE_NOALLOC_MAX_POINTS); use rd_decimate";
        return report_error(RD_ERR_CAPACITY, msg.c_str());
    }
    int32_t* scratch = nullptr;
    cudaError_t e = scratch_on_current_device(&scratch);
    if (e != cudaSuccess)
        return report_error(RD_ERR_CUDA, (std::string("cudaGetSymbolAddress: ") +
                                          cudaGetErrorString(e)).c_str());
    if (dim == 2) k_decimate_noalloc<2, 512><<<1, 512, 0, st>>>(d_S, (int)ns, r2, d_ns_out, scratch);
    else k_decimate_noalloc<3, 512><<<1, 512, 0, st>>>(d_S, (int)ns, r2, d_ns_out, scratch);
    e = cudaGetLastError();
    if (e != cudaSuccess)
        return report_error(RD_ERR_CUDA, (std::string("launch: ") + cudaGetErrorString(e)).c_str());
    return RD_OK;
}

}  // namespace rdb
