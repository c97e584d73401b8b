// rd_internal.cuh -- shared device-side definitions of the B200 ridge-detection
// engine: per-cloud descriptors, exact FP32 arithmetic helpers and error bits.
//
// Exactness contract.  Every floating-point result that decides a discrete
// outcome (a choose, an assignment, a movement test, a decimation count) or that
// is written back as a chosen coordinate is computed with explicitly rounded
// intrinsics (__fsub_rn/__fmul_rn/__fadd_rn/__fdiv_rn), in the operation order of
// the reference CPU code, so nvcc cannot contract a multiply and an add into an
// FMA.  With that, the GPU path reproduces the reference's serial CPU output bit
// for bit:
//   squared distance   t = a - b; acc += t*t, d = 0..DIM-1    rd/cpu/brute_force/rd_inner.hpp:42-49
//   argmin             strict '<', lowest index wins ties     rd/cpu/brute_force/evolve.hpp:54-65
//   membership         min <= r1*r1                            rd/cpu/brute_force/evolve.hpp:66
//   centroid sums      FP32, in cloud-point index order        rd/cpu/brute_force/evolve.hpp:66-75
//   shift test         |mc - c| > 2.f*|mc|*cnt*FLT_EPSILON     rd/cpu/brute_force/evolve.hpp:151-153
#pragma once

#include <cfloat>
#include <cstdint>
#include <cuda_runtime.h>
#include <type_traits>

namespace rdb {

// Point dimensions built into the kernels: 1 to RD_MAX_DIM (the reference's
// CPU path takes the dimension at run time, its GPU classes as a template
// argument).  with_dim calls f(std::integral_constant<int, DIM>) for a
// supported dim and returns cudaErrorInvalidValue otherwise.
constexpr int RD_MAX_DIM = 4;
__host__ __device__ constexpr bool dim_supported(int dim) { return dim >= 1 && dim <= RD_MAX_DIM; }

template <class F>
inline cudaError_t with_dim(int dim, F&& f)
{
    switch (dim) {
        case 1: return f(std::integral_constant<int, 1>{});
        case 2: return f(std::integral_constant<int, 2>{});
        case 3: return f(std::integral_constant<int, 3>{});
        case 4: return f(std::integral_constant<int, 4>{});
        default: return cudaErrorInvalidValue;
    }
}

// ---------------------------------------------------------------------------
// error bits recorded on the device (per cloud and globally); the host turns
// them into rd_status codes.  No kernel ever traps.
// ---------------------------------------------------------------------------
enum : int {
    ERRB_EVOLVE_CAP = 1 << 0,   // evolve pass limit reached before convergence
    ERRB_OUTER_CAP = 1 << 1,    // outer (evolve/decimate) iteration limit reached
    ERRB_CAPACITY = 1 << 2,     // a device buffer would have overflowed
    ERRB_DEC_CAP = 1 << 3,      // decimation pass limit reached
};

// phases of one cloud's state machine
enum : int {
    PH_EVOLVE = 0,      // evolve passes running
    PH_CONVERGED = 1,   // evolve converged, waiting for its group's decimation
    PH_DONE = 2,        // chosen count stable: finished
};

// Per-cloud descriptor.  A "cloud" is a set of evolve points with its own chosen
// set: a whole input cloud for the brute-force and batched paths, or one leaf
// tile (own points first, then its r1 halo) for the tiled path.  Clouds of one
// group are decimated together (a tiled run is a single group; every
// brute-force cloud is its own group).
struct CloudDesc {
    int64_t p_off;       // first point slot of this cloud in the packed point array
    int32_t n_all;       // evolve points (own + halo)
    int32_t n_own;       // choose points (own points; == n_all for brute force)
    float r1, r2;
    int64_t s_off;       // first chosen slot (capacity n_own)
    int64_t chunk_begin; // first assignment chunk of this cloud
    int32_t n_chunks;
    int32_t group;
    int64_t hist_off;    // start of this cloud's chunk x key histogram (set after choose)
    int32_t ns_cap;      // chosen count right after choose (hist row length)
    int64_t key_off;     // start of this cloud's per-chosen arrays (cnt/base)
    int64_t hash_off;    // start of this cloud's choose hash heads
    int32_t hash_bits;   // log2 of the number of hash buckets
    int32_t pad;
};

struct GroupDesc {
    int32_t cloud_begin;
    int32_t n_clouds;
    int32_t nocopy;      // decimateNoCopy semantics (tiled) instead of decimate
    int32_t s_cap;       // scratch slots of the group (its members' chosen capacity)
    int64_t s_scratch;   // first scratch slot of the group's decimation
};

// coordinates per point in padded device copies: DIM 3 is stored as float4
template <int DIM>
struct PadDim { static constexpr int v = (DIM == 3) ? 4 : DIM; };
inline int pad_dim(int dim) { return dim == 3 ? 4 : dim; }

// slot-order chunk of position i of a cloud of n points in m chunks: the lc
// with floor(lc n / m) <= i < floor((lc + 1) n / m), i.e. lc n < (i + 1) m <=
// (lc + 1) n; a float estimate corrected with exact integer products
__device__ __forceinline__ int slot_chunk(int i, int n, int m, float ratio)
{
    int lc = min(max(__float2int_rz(__fmul_rn((float)i, ratio)), 0), m - 1);
    const int64_t t = (int64_t)(i + 1) * m;
    while (lc > 0 && (int64_t)lc * n >= t) --lc;
    while (lc < m - 1 && (int64_t)(lc + 1) * n < t) ++lc;
    return lc;
}

constexpr int KBLK = 32;  // chosen points per histogram-scan block (one per lane)

// ---------------------------------------------------------------------------
// exact FP32 helpers
// ---------------------------------------------------------------------------
template <int DIM>
__device__ __forceinline__ float sqdist_exact(const float* a, const float* b)
{
    float t = __fsub_rn(a[0], b[0]);
    float acc = __fmul_rn(t, t);  // 0 + t*t == t*t exactly
#pragma unroll
    for (int d = 1; d < DIM; ++d) {
        t = __fsub_rn(a[d], b[d]);
        acc = __fadd_rn(acc, __fmul_rn(t, t));
    }
    return acc;
}

// The same distance for two points at once: differences and squares on the
// packed FP32 pipe of sm_100 (each lane of __fadd2_rn / __fmul2_rn rounds like
// the scalar op; np[d] holds (-p0[d], -p1[d]) and s + (-p) == s - p exactly),
// the accumulation in scalar adds.  A packed add whose operand is a packed
// product is fused into a packed FMA by the compiler even with contraction
// disabled, which would change the rounding; scalar adds of the product
// lanes are not.
template <int DIM>
__device__ __forceinline__ float2 sqdist2_exact(const float* s, const float2* np)
{
    float2 t = __fadd2_rn(make_float2(s[0], s[0]), np[0]);
    const float2 q0 = __fmul2_rn(t, t);
    float a0 = q0.x, a1 = q0.y;
#pragma unroll
    for (int d = 1; d < DIM; ++d) {
        t = __fadd2_rn(make_float2(s[d], s[d]), np[d]);
        const float2 q = __fmul2_rn(t, t);
        a0 = __fadd_rn(a0, q.x);
        a1 = __fadd_rn(a1, q.y);
    }
    return make_float2(a0, a1);
}

__device__ __forceinline__ float sqr_rn(float r) { return __fmul_rn(r, r); }

// Cells of the spatial order used by the culled assignment: cell coordinate
// floor(x * inv) with inv = 4 / r1 (edge r1/4), wrapped to 32 bits;
// non-finite or huge coordinates land in cell 0.  The order only changes how
// tight the culling boxes are, never a result.
__device__ __forceinline__ float spatial_cell_inv(float r1) { return 4.0f / r1; }

__device__ __forceinline__ uint32_t spatial_cell(float x, float inv)
{
    const float f = floorf(x * inv);
    if (!(f > -1.0e15f && f < 1.0e15f)) return 0u;
    return (uint32_t)(uint64_t)(int64_t)f;
}


// Runs of equal keys of a warp, for stable grouping without match
// instructions (the match instruction's throughput drops when a warp holds
// many distinct keys, as in a brute-force cloud visited in random order): the 32 (key, lane) pairs are sorted by key, ties by lane
// (a bitonic network of shuffles); lane p then holds the p-th element of that
// order.  key < 0 means "no key" and sorts last.  Keys must be < 2^26.
struct WarpRun {
    int key;      // key of the element held (-1: none)
    int src;      // its lane before the sort
    int rank;     // its position among the elements of its key (in lane order)
    int count;    // elements of its key in the warp
    int head;     // lane holding the first element of its key
};

__device__ __forceinline__ WarpRun warp_runs(const int key, const int lane)
{
    constexpr unsigned NONE = 0x3FFFFFFu;
    unsigned v = ((key < 0 ? NONE : (unsigned)key) << 5) | (unsigned)lane;
#pragma unroll
    for (int k = 2; k <= 32; k <<= 1) {
#pragma unroll
        for (int j = k >> 1; j > 0; j >>= 1) {
            const unsigned o = __shfl_xor_sync(0xffffffffu, v, j);
            const bool up = (lane & k) == 0 || k == 32;
            const bool lower = (lane & j) == 0;
            v = (lower == up) ? min(v, o) : max(v, o);
        }
    }
    WarpRun r;
    const unsigned ks = v >> 5;
    r.src = (int)(v & 31u);
    r.key = (ks == NONE) ? -1 : (int)ks;
    const unsigned prev = __shfl_up_sync(0xffffffffu, ks, 1);
    const unsigned heads = __ballot_sync(0xffffffffu, lane == 0 || prev != ks);
    const unsigned le = (lane == 31) ? 0xffffffffu : ((2u << lane) - 1u);
    r.head = 31 - __clz(heads & le);
    const unsigned after = heads & ~le;
    const int end = after ? (__ffs(after) - 1) : 32;
    r.rank = lane - r.head;
    r.count = end - r.head;
    return r;
}


// shift of one coordinate (rd/cpu/brute_force/evolve.hpp:143-177); returns 1
// when the coordinate moved.
__device__ __forceinline__ int shift_coord(float sum, int cnt, float& c)
{
    const float fc = (float)cnt;
    const float mc = __fdiv_rn(sum, fc);
    float thr = __fmul_rn(2.0f, fabsf(mc));
    thr = __fmul_rn(thr, fc);
    thr = __fmul_rn(thr, FLT_EPSILON);
    if (fabsf(__fsub_rn(mc, c)) > thr) {
        c = mc;
        return 1;
    }
    return 0;
}

__device__ __forceinline__ unsigned lanemask_lt()
{
    unsigned m;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

}  // namespace rdb
