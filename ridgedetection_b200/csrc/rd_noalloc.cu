// rd_noalloc.cu -- decimation that allocates no device memory.
//
// Some callers cannot call cudaMalloc: code that runs while a CUDA graph is
// being captured (an allocation would break the capture), real-time or
// embedded hosts that forbid allocation after start-up, and plugins whose
// device memory is owned by a framework that does not hand out a workspace.
// rd_decimate_noalloc serves them: its scratch lives in one file-scope
// __device__ array of fixed size, so a call only launches kernels.
//
// The array is RD_DECIMATE_NOALLOC_SCRATCH_BYTES (about 1.4 MB) on every GPU
// that loads the library, held until the process exits.  Every call uses the
// same array: two calls whose kernels overlap on the GPU (different streams,
// or different host threads) race on it.  Each call clears what must start
// at zero (bucket counts, error flag) and overwrites the rest before reading.
#include "../../include/rd_c_api.h"
#include "rd_grid.cuh"

#include <mutex>
#include <string>

namespace rdb {

const char* noalloc_error_message = nullptr;  // set on failure; read by rd_capi.cu

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
int32_t* g_dev_ptr[MAX_DEVICES] = {};

// Device address of the scratch on the current device, looked up once per
// device with that device current.
cudaError_t scratch_on_current_device(int32_t** out)
{
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= MAX_DEVICES) return cudaErrorInvalidDevice;
    std::lock_guard<std::mutex> lk(g_mu);
    if (!g_dev_ptr[dev]) {
        void* p = nullptr;
        e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess) return e;
        g_dev_ptr[dev] = static_cast<int32_t*>(p);
    }
    *out = g_dev_ptr[dev];
    return cudaSuccess;
}

}  // namespace

int decimate_noalloc(int dim, float* d_S, int64_t ns, float r2, int32_t* d_ns_out,
                     cudaStream_t st)
{
    static thread_local std::string msg;
    if (dim != 2 && dim != 3) { msg = "dim must be 2 or 3"; noalloc_error_message = msg.c_str(); return RD_ERR_UNSUPPORTED; }
    if (!d_S || !d_ns_out || ns < 0 || !(r2 > 0.0f)) {
        msg = "null pointer, negative count or r2 <= 0";
        noalloc_error_message = msg.c_str();
        return RD_ERR_ARG;
    }
    if (ns > NA_MAX) {
        msg = "rd_decimate_noalloc: " + std::to_string(ns) + " points exceed the fixed scratch limit of " +
              std::to_string(NA_MAX) + " (RD_DECIMATE_NOALLOC_MAX_POINTS); use rd_decimate";
        noalloc_error_message = msg.c_str();
        return RD_ERR_CAPACITY;
    }
    int32_t* scratch = nullptr;
    cudaError_t e = scratch_on_current_device(&scratch);
    if (e != cudaSuccess) {
        msg = std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e);
        noalloc_error_message = msg.c_str();
        return RD_ERR_CUDA;
    }
    if (dim == 2) k_decimate_noalloc<2, 512><<<1, 512, 0, st>>>(d_S, (int)ns, r2, d_ns_out, scratch);
    else k_decimate_noalloc<3, 512><<<1, 512, 0, st>>>(d_S, (int)ns, r2, d_ns_out, scratch);
    e = cudaGetLastError();
    if (e != cudaSuccess) {
        msg = std::string("launch: ") + cudaGetErrorString(e);
        noalloc_error_message = msg.c_str();
        return RD_ERR_CUDA;
    }
    return RD_OK;
}

}  // namespace rdb
