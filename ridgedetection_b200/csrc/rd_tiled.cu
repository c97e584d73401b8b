// rd_tiled.cu -- tile build and driver of the extended-tile tiled variant
// (see rd_tiled.hpp for the semantics and the reference citations).
#include "rd_tiled.hpp"

#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>

namespace rdb {

namespace {

constexpr int MAXD = RD_MAX_DIM;

__device__ __forceinline__ int f2s(float f)
{
    const int i = __float_as_int(f);
    return i >= 0 ? i : i ^ 0x7FFFFFFF;
}
__host__ __device__ inline float s2f(int s)
{
    const int i = s >= 0 ? s : s ^ 0x7FFFFFFF;
    float f;
    std::memcpy(&f, &i, 4);
    return f;
}

__global__ void k_bbox_init(int* box, int dim)
{
    const int d = threadIdx.x;
    if (d < dim) {
        box[2 * d] = 0x7FFFFFFF;
        box[2 * d + 1] = (int)0x80000000;
    }
}

// rd/utils/bounding_box.hpp:126-197: per-dimension min and max (exact)
template <int DIM>
__global__ void __launch_bounds__(256) k_bbox(const float* __restrict__ P, int64_t n, int* box)
{
    __shared__ int smin[DIM], smax[DIM];
    if (threadIdx.x < DIM) {
        smin[threadIdx.x] = 0x7FFFFFFF;
        smax[threadIdx.x] = (int)0x80000000;
    }
    __syncthreads();
    int lmin[DIM], lmax[DIM];
#pragma unroll
    for (int d = 0; d < DIM; ++d) { lmin[d] = 0x7FFFFFFF; lmax[d] = (int)0x80000000; }
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
#pragma unroll
        for (int d = 0; d < DIM; ++d) {
            const int s = f2s(P[i * DIM + d]);
            lmin[d] = min(lmin[d], s);
            lmax[d] = max(lmax[d], s);
        }
    }
#pragma unroll
    for (int d = 0; d < DIM; ++d) {
        atomicMin(&smin[d], lmin[d]);
        atomicMax(&smax[d], lmax[d]);
    }
    __syncthreads();
    if (threadIdx.x < DIM) {
        atomicMin(&box[2 * threadIdx.x], smin[threadIdx.x]);
        atomicMax(&box[2 * threadIdx.x + 1], smax[threadIdx.x]);
    }
}

// Per-dimension tile bounds: tmin[off[d] + c], tmax[off[d] + c]
struct GridDesc {
    int n[MAXD];
    int off[MAXD];
    float gmin[MAXD];
    float step[MAXD];
    float r;
};

// ext-containing and own tile intervals of coordinate x along one dimension
__device__ __forceinline__ void dim_ranges(float x, int d, const GridDesc& g,
                                           const float* __restrict__ tmin,
                                           const float* __restrict__ tmax, int& lo, int& hi,
                                           int& own)
{
    const int n = g.n[d];
    int a = 0, b = n - 1;
    if (g.step[d] > 0.0f) {
        const double s = (double)g.step[d];
        const double c0 = floor(((double)x - (double)g.gmin[d]) / s);
        const double m = ceil((double)g.r / s) + 2.0;
        const double fa = fmax(c0 - m, 0.0), fb = fmin(c0 + m, (double)(n - 1));
        a = (int)fa;
        b = (int)fb;
        if (a > b) { a = 0; b = -1; }
    }
    lo = n;
    hi = -1;
    own = -1;
    const float* mn = tmin + g.off[d];
    const float* mx = tmax + g.off[d];
    for (int c = a; c <= b; ++c) {
        const float emin = __fsub_rn(mn[c], g.r);
        const float emax = __fadd_rn(mx[c], g.r);
        if (!(x < emin) && !(x >= emax)) {
            lo = min(lo, c);
            hi = max(hi, c);
        }
        if (!(x < mn[c]) && !(x >= mx[c])) own = c;
    }
}

template <int DIM>
__global__ void __launch_bounds__(256) k_emit_count(const float* __restrict__ P, int64_t n,
                                                    GridDesc g, const float* __restrict__ tmin,
                                                    const float* __restrict__ tmax,
                                                    int32_t* __restrict__ cnt)
{
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        int prod = 1;
#pragma unroll
        for (int d = 0; d < DIM; ++d) {
            int lo, hi, own;
            dim_ranges(P[i * DIM + d], d, g, tmin, tmax, lo, hi, own);
            prod *= (hi >= lo) ? (hi - lo + 1) : 0;
        }
        cnt[i] = prod;
    }
}

// emission in point order: own tile (key 2t) first, then halo tiles (key 2t+1)
template <int DIM>
__global__ void __launch_bounds__(256) k_emit_fill(const float* __restrict__ P, int64_t n,
                                                   GridDesc g, const float* __restrict__ tmin,
                                                   const float* __restrict__ tmax,
                                                   const int32_t* __restrict__ off,
                                                   uint32_t* __restrict__ keys,
                                                   int32_t* __restrict__ vals)
{
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        int lo[DIM], hi[DIM], own[DIM];
        bool any = true, inside = true;
#pragma unroll
        for (int d = 0; d < DIM; ++d) {
            dim_ranges(P[i * DIM + d], d, g, tmin, tmax, lo[d], hi[d], own[d]);
            any = any && (hi[d] >= lo[d]);
            inside = inside && (own[d] >= 0);
        }
        if (!any) continue;
        int w = off[i];
        int town = -1;
        if (inside) {
            int t = 0, mul = 1;
#pragma unroll
            for (int d = 0; d < DIM; ++d) { t += own[d] * mul; mul *= g.n[d]; }
            town = t;
            keys[w] = 2u * (uint32_t)t;
            vals[w] = (int32_t)i;
            ++w;
        }
        int c[DIM];
#pragma unroll
        for (int d = 0; d < DIM; ++d) c[d] = lo[d];
        for (;;) {
            int t = 0, mul = 1;
#pragma unroll
            for (int d = 0; d < DIM; ++d) { t += c[d] * mul; mul *= g.n[d]; }
            if (t != town) {
                keys[w] = 2u * (uint32_t)t + 1u;
                vals[w] = (int32_t)i;
                ++w;
            }
            int d = 0;
            for (; d < DIM; ++d) {
                if (c[d] < hi[d]) { ++c[d]; break; }
                c[d] = lo[d];
            }
            if (d == DIM) break;
        }
    }
}

__global__ void k_seg_bounds(const uint32_t* __restrict__ keys, int64_t m, int32_t* seg)
{
    for (int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; j < m;
         j += (int64_t)gridDim.x * blockDim.x) {
        const uint32_t k = keys[j];
        if (j == 0 || keys[j - 1] != k) seg[2 * k] = (int32_t)j;
        if (j == m - 1 || keys[j + 1] != k) seg[2 * k + 1] = (int32_t)(j + 1);
    }
}

template <int DIM>
__global__ void k_gather_idx(const float* __restrict__ P, const int32_t* __restrict__ idx,
                             int64_t m, float* __restrict__ out)
{
    for (int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; j < m * DIM;
         j += (int64_t)gridDim.x * blockDim.x) {
        const int64_t s = j / DIM;
        const int d = (int)(j - s * DIM);
        out[j] = P[(int64_t)idx[s] * DIM + d];
    }
}

// ---------------------------------------------------------------------------
// Subdivision of oversize tiles on the device, one level at a time
// (grouped_tile_tree.inl:247-330).  A level holds nodes; node i's entries are
// its own points then its halo points (code = 2 i + 0 / 1).  Each node is cut
// in two halves along one dimension (boxes from the host, computed with the
// reference's FP32 operations); an own point goes to the own list of the first
// half that contains it and to the halo list of every half it is near; a halo
// point to the halo lists it is near.  Outputs are (key, point) pairs with key
// = 2 (2 i + s) + (0 own / 1 halo), sorted stably, so every list keeps the
// parent's order (own-derived halo entries before halo-derived ones).
// ---------------------------------------------------------------------------
struct SplitBox {
    float mn[2][MAXD], mx[2][MAXD], emin[2][MAXD], emax[2][MAXD];
};

// own: mn <= x < mx in every dimension; halo ("nearby"): inside the box
// grown by r1 on every side (emin = mn - r1, emax = mx + r1, FP32) but not
// own -- the tests of grouped_tile_tree.inl's isInside / isNearby
template <int DIM>
__device__ __forceinline__ void split_flags(const float* p, const SplitBox& b, const int kind,
                                            int& own_s, bool (&near)[2])
{
    own_s = -1;
#pragma unroll
    for (int s = 0; s < 2; ++s) {
        bool in = true, nb = true;
#pragma unroll
        for (int d = 0; d < DIM; ++d) {
            if (p[d] < b.mn[s][d] || p[d] >= b.mx[s][d]) in = false;
            if (p[d] < b.emin[s][d] || p[d] >= b.emax[s][d]) nb = false;
        }
        near[s] = nb && !in;
        if (kind == 0 && in && own_s < 0) own_s = s;
    }
}

template <int DIM>
__global__ void __launch_bounds__(256) k_split_count(const float* __restrict__ P,
                                                     const int32_t* __restrict__ E,
                                                     const int32_t* __restrict__ code, int64_t nE,
                                                     const SplitBox* __restrict__ boxes,
                                                     int32_t* __restrict__ cnt)
{
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < nE;
         e += (int64_t)gridDim.x * blockDim.x) {
        float p[DIM];
#pragma unroll
        for (int d = 0; d < DIM; ++d) p[d] = P[(int64_t)E[e] * DIM + d];
        int own_s;
        bool near[2];
        split_flags<DIM>(p, boxes[code[e] >> 1], code[e] & 1, own_s, near);
        cnt[e] = (own_s >= 0) + (int)near[0] + (int)near[1];
    }
}

template <int DIM>
__global__ void __launch_bounds__(256) k_split_fill(const float* __restrict__ P,
                                                    const int32_t* __restrict__ E,
                                                    const int32_t* __restrict__ code, int64_t nE,
                                                    const SplitBox* __restrict__ boxes,
                                                    const int32_t* __restrict__ off,
                                                    uint32_t* __restrict__ keys,
                                                    int32_t* __restrict__ vals)
{
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < nE;
         e += (int64_t)gridDim.x * blockDim.x) {
        float p[DIM];
        const int32_t i = E[e];
#pragma unroll
        for (int d = 0; d < DIM; ++d) p[d] = P[(int64_t)i * DIM + d];
        const int node = code[e] >> 1;
        int own_s;
        bool near[2];
        split_flags<DIM>(p, boxes[node], code[e] & 1, own_s, near);
        int o = off[e];
        if (own_s >= 0) {
            keys[o] = (uint32_t)(2 * (2 * node + own_s));
            vals[o++] = i;
        }
#pragma unroll
        for (int s = 0; s < 2; ++s)
            if (near[s]) {
                keys[o] = (uint32_t)(2 * (2 * node + s) + 1);
                vals[o++] = i;
            }
    }
}

// gathers the entries of the nodes of a level: tab per node = (first source
// entry, entries, first destination entry); entries get code 2 node + kind,
// kind = 1 from own_n on (the node's own points come first)
__global__ void k_split_seed(const int32_t* __restrict__ src, const int64_t* __restrict__ tab,
                             int nnodes, int32_t* __restrict__ E, int32_t* __restrict__ code)
{
    for (int q = blockIdx.y; q < nnodes; q += gridDim.y) {
        const int64_t so = tab[4 * q], nn = tab[4 * q + 1], own_n = tab[4 * q + 2],
                      dof = tab[4 * q + 3];
        for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < nn;
             e += (int64_t)gridDim.x * blockDim.x) {
            E[dof + e] = src[so + e];
            code[dof + e] = 2 * q + (e >= own_n ? 1 : 0);
        }
    }
}

// leaf chosen points -> one array in leaf order; tab: (src float off, n floats, dst float off)
__global__ void k_concat(const float* __restrict__ S, const int64_t* __restrict__ tab, int nl,
                         float* __restrict__ out)
{
    for (int l = blockIdx.y; l < nl; l += gridDim.y) {
        const int64_t so = tab[3 * l], nf = tab[3 * l + 1], dof = tab[3 * l + 2];
        for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < nf;
             e += (int64_t)gridDim.x * blockDim.x)
            out[dof + e] = S[so + e];
    }
}

int grid_of(int64_t n) { return (int)std::max<int64_t>(1, std::min<int64_t>((n + 255) / 256, 148 * 32)); }

// ---------------------------------------------------------------------------
// host-side tile geometry, identical FP32 operations to the reference
// ---------------------------------------------------------------------------
struct HBox {
    float mn[MAXD], mx[MAXD], dist[MAXD];
};

// rd/utils/bounding_box.hpp:210-227
void calc_dist(HBox& b, int dim)
{
    for (int d = 0; d < dim; ++d) {
        const float x = std::fabs(b.mx[d] - b.mn[d]);
        b.dist[d] = (x <= FLT_EPSILON) ? 0.0f : x;
    }
}

// grouped_tile_tree.inl:147-213 for one dimension: bounds of tile c of n
void tile_bounds(const HBox& p, int d, int c, int n, float& mn, float& mx)
{
    const float step = p.dist[d] / (float)n;
    const volatile float lo = (float)c * step;
    const volatile float hi = (float)(c + 1) * step;
    mn = p.mn[d] + lo;
    mx = p.mn[d] + hi;
    if (c == n - 1) mx = p.mx[d];
}

}  // namespace

int TiledRunner::fail(const char* what, cudaError_t e)
{
    last_error = std::string(what) + ": " + cudaGetErrorString(e);
    return 2;
}

#define TK(call)                                      \
    do {                                              \
        cudaError_t e_ = (call);                      \
        if (e_ != cudaSuccess) return fail(#call, e_); \
    } while (0)

int TiledRunner::run(const float* d_points, int64_t n, int dim, float r1, float r2, int64_t cap,
                     const int32_t* tpd, bool use_graph, cudaStream_t st)
{
    using clk = std::chrono::steady_clock;
    const auto t0 = clk::now();
    tm_ = TiledTimers();
    ns_ = 0;
    leaf_ns_.clear();
    if (!dim_supported(dim)) { last_error = "dim must be 1 to 4"; return 6; }
    if (n <= 0) return 0;
    if (n > INT32_MAX / 4) { last_error = "too many points"; return 1; }
    int64_t ntiles = 1;
    for (int d = 0; d < dim; ++d) {
        if (tpd[d] < 1) { last_error = "tiles_per_dim must be >= 1"; return 1; }
        ntiles *= tpd[d];
    }
    if (ntiles > (1 << 26)) { last_error = "too many tiles"; return 1; }

    // 1. bounding box
    TK(bBox_.ensure(8 * MAXD));
    k_bbox_init<<<1, 32, 0, st>>>(bBox_.as<int>(), dim);
    TK(with_dim(dim, [&](auto D) {
        k_bbox<decltype(D)::value><<<grid_of(n), 256, 0, st>>>(d_points, n, bBox_.as<int>());
        return cudaGetLastError();
    }));
    int hbox[2 * MAXD];
    TK(cudaMemcpyAsync(hbox, bBox_.p, 8 * dim, cudaMemcpyDeviceToHost, st));
    TK(cudaStreamSynchronize(st));
    HBox g;
    for (int d = 0; d < dim; ++d) {
        g.mn[d] = s2f(hbox[2 * d]);
        g.mx[d] = s2f(hbox[2 * d + 1]);
    }
    calc_dist(g, dim);

    // 2. root tile bounds per dimension (grouped_tile_tree.inl:147-213)
    GridDesc gd;
    std::memset(&gd, 0, sizeof(gd));
    std::vector<float> hb;
    int tot = 0;
    for (int d = 0; d < dim; ++d) tot += tpd[d];
    hb.resize(2 * tot);
    int off = 0;
    for (int d = 0; d < dim; ++d) {
        gd.n[d] = tpd[d];
        gd.off[d] = off;
        gd.gmin[d] = g.mn[d];
        gd.step[d] = g.dist[d] / (float)tpd[d];
        for (int c = 0; c < tpd[d]; ++c)
            tile_bounds(g, d, c, tpd[d], hb[off + c], hb[tot + off + c]);
        off += tpd[d];
    }
    gd.r = r1;
    TK(bBounds_.ensure(sizeof(float) * hb.size()));
    TK(cudaMemcpyAsync(bBounds_.p, hb.data(), sizeof(float) * hb.size(), cudaMemcpyHostToDevice,
                       st));
    const float* tmin = bBounds_.as<float>();
    const float* tmax = tmin + tot;

    // 3. emission counts and offsets (point order)
    TK(bCnt_.ensure(4 * (size_t)(n + 1)));
    TK(bOff_.ensure(4 * (size_t)(n + 1)));
    TK(with_dim(dim, [&](auto D) {
        k_emit_count<decltype(D)::value><<<grid_of(n), 256, 0, st>>>(d_points, n, gd, tmin, tmax,
                                                                    bCnt_.as<int32_t>());
        return cudaGetLastError();
    }));
    size_t tb = 0;
    TK(cub::DeviceScan::ExclusiveSum(nullptr, tb, bCnt_.as<int32_t>(), bOff_.as<int32_t>(), (int)n, st));
    TK(bTemp_.ensure(tb));
    TK(cub::DeviceScan::ExclusiveSum(bTemp_.p, tb, bCnt_.as<int32_t>(), bOff_.as<int32_t>(), (int)n, st));
    int32_t last_off = 0, last_cnt = 0;
    TK(cudaMemcpyAsync(&last_off, bOff_.as<int32_t>() + n - 1, 4, cudaMemcpyDeviceToHost, st));
    TK(cudaMemcpyAsync(&last_cnt, bCnt_.as<int32_t>() + n - 1, 4, cudaMemcpyDeviceToHost, st));
    TK(cudaStreamSynchronize(st));
    const int64_t m = (int64_t)last_off + last_cnt;

    // 4. emit (key, point) pairs and sort them stably by key
    TK(bKeys_.ensure(4 * (size_t)(m + 1)));
    TK(bVals_.ensure(4 * (size_t)(m + 1)));
    TK(bKeys2_.ensure(4 * (size_t)(m + 1)));
    TK(bVals2_.ensure(4 * (size_t)(m + 1)));
    TK(with_dim(dim, [&](auto D) {
        k_emit_fill<decltype(D)::value><<<grid_of(n), 256, 0, st>>>(
            d_points, n, gd, tmin, tmax, bOff_.as<int32_t>(), bKeys_.as<uint32_t>(),
            bVals_.as<int32_t>());
        return cudaGetLastError();
    }));
    int bits = 1;
    while ((int64_t(1) << bits) < 2 * ntiles) ++bits;
    tb = 0;
    TK(cub::DeviceRadixSort::SortPairs(nullptr, tb, bKeys_.as<uint32_t>(), bKeys2_.as<uint32_t>(),
                                       bVals_.as<int32_t>(), bVals2_.as<int32_t>(), (int)m, 0, bits,
                                       st));
    TK(bTemp_.ensure(tb));
    TK(cub::DeviceRadixSort::SortPairs(bTemp_.p, tb, bKeys_.as<uint32_t>(), bKeys2_.as<uint32_t>(),
                                       bVals_.as<int32_t>(), bVals2_.as<int32_t>(), (int)m, 0, bits,
                                       st));
    // 5. per-key segments
    TK(bSeg_.ensure(8 * (size_t)(2 * ntiles + 1)));
    TK(cudaMemsetAsync(bSeg_.p, 0, 8 * (size_t)(2 * ntiles), st));
    k_seg_bounds<<<grid_of(m), 256, 0, st>>>(bKeys2_.as<uint32_t>(), m, bSeg_.as<int32_t>());
    TK(cudaGetLastError());
    std::vector<int32_t> seg(4 * ntiles);
    TK(cudaMemcpyAsync(seg.data(), bSeg_.p, 4 * seg.size(), cudaMemcpyDeviceToHost, st));
    TK(cudaStreamSynchronize(st));

    // 6. leaves in pre-order.  Tiles with cap or more own points are split on
    //    the device, level by level (k_split_*); their leaves take the tile's
    //    place in the pre-order, ordered by their split paths.
    std::vector<CloudDesc> cl;
    auto own_of = [&](int64_t t, int64_t& s, int64_t& e) { s = seg[4 * t]; e = seg[4 * t + 1]; };
    auto halo_of = [&](int64_t t, int64_t& s, int64_t& e) { s = seg[4 * t + 2]; e = seg[4 * t + 3]; };
    struct SubLeaf {
        int64_t root;
        uint64_t path;     // split choices, left-aligned: pre-order = increasing path
        int buf;           // level buffer holding its lists
        int64_t off, own, halo;
    };
    struct SplitNode {
        HBox box;
        int64_t root;
        uint64_t path;
        int depth;         // splits above it (its level is depth + 1)
        int64_t src, own, halo;  // its lists in the current source buffer
    };
    std::vector<SubLeaf> subleaves;
    std::vector<SplitNode> nodes;
    for (int64_t t = 0; t < ntiles; ++t) {
        int64_t os, oe, hs, he;
        own_of(t, os, oe);
        halo_of(t, hs, he);
        const int64_t no = oe - os, nh = he - hs;
        if (nh > 0 && no > 0 && hs != oe) { last_error = "internal: tile segments not adjacent"; return 2; }
        if (no <= 1 || no < cap) continue;
        SplitNode nd;
        int64_t rem = t;
        for (int d = 0; d < dim; ++d) {
            const int c = (int)(rem % tpd[d]);
            rem /= tpd[d];
            nd.box.mn[d] = hb[gd.off[d] + c];
            nd.box.mx[d] = hb[tot + gd.off[d] + c];
        }
        calc_dist(nd.box, dim);
        nd.root = t;
        nd.path = 0;
        nd.depth = 0;
        nd.src = os;
        nd.own = no;
        nd.halo = nh;
        nodes.push_back(nd);
    }
    split_bufs_.clear();
    const int32_t* src_vals = bVals2_.as<int32_t>();
    while (!nodes.empty()) {
        const int nn = (int)nodes.size();
        if (nodes[0].depth + 1 > 64) {
            last_error = "tile subdivision did not terminate (duplicate points above capacity)";
            return 1;
        }
        // this level's entries and the two halves of every node
        std::vector<int64_t> tab(4 * (size_t)nn);
        std::vector<SplitBox> boxes((size_t)nn);
        std::vector<HBox> halves(2 * (size_t)nn);
        int64_t nE = 0;
        for (int q = 0; q < nn; ++q) {
            const SplitNode& nd = nodes[q];
            tab[4 * q] = nd.src;
            tab[4 * q + 1] = nd.own + nd.halo;
            tab[4 * q + 2] = nd.own;
            tab[4 * q + 3] = nE;
            nE += nd.own + nd.halo;
            const int sd = (nd.depth + 1) % dim;
            for (int sh = 0; sh < 2; ++sh) {
                HBox& hbx = halves[2 * q + sh];
                for (int d = 0; d < dim; ++d) {
                    if (d == sd) tile_bounds(nd.box, d, sh, 2, hbx.mn[d], hbx.mx[d]);
                    else tile_bounds(nd.box, d, 0, 1, hbx.mn[d], hbx.mx[d]);
                }
                calc_dist(hbx, dim);
                for (int d = 0; d < MAXD; ++d) {
                    const bool live = d < dim;
                    boxes[q].mn[sh][d] = live ? hbx.mn[d] : 0.0f;
                    boxes[q].mx[sh][d] = live ? hbx.mx[d] : 0.0f;
                    const volatile float emin = live ? hbx.mn[d] - r1 : 0.0f;
                    const volatile float emax = live ? hbx.mx[d] + r1 : 0.0f;
                    boxes[q].emin[sh][d] = emin;
                    boxes[q].emax[sh][d] = emax;
                }
            }
        }
        if (nE > INT32_MAX / 4) { last_error = "subdivision level too large"; return 1; }
        TK(bSplitTab_.ensure(sizeof(int64_t) * tab.size()));
        TK(cudaMemcpyAsync(bSplitTab_.p, tab.data(), sizeof(int64_t) * tab.size(),
                           cudaMemcpyHostToDevice, st));
        TK(bSplitBox_.ensure(sizeof(SplitBox) * boxes.size()));
        TK(cudaMemcpyAsync(bSplitBox_.p, boxes.data(), sizeof(SplitBox) * boxes.size(),
                           cudaMemcpyHostToDevice, st));
        TK(bSplitE_.ensure(4 * (size_t)(nE + 1)));
        TK(bSplitCode_.ensure(4 * (size_t)(nE + 1)));
        TK(bSplitCnt_.ensure(4 * (size_t)(nE + 1)));
        TK(bSplitOff_.ensure(4 * (size_t)(nE + 1)));
        {
            dim3 g((unsigned)std::min<int64_t>(64, (nE + 255) / 256 + 1), (unsigned)std::min(nn, 1024));
            k_split_seed<<<g, 256, 0, st>>>(src_vals, bSplitTab_.as<int64_t>(), nn,
                                            bSplitE_.as<int32_t>(), bSplitCode_.as<int32_t>());
            TK(cudaGetLastError());
        }
        TK(with_dim(dim, [&](auto D) {
            k_split_count<decltype(D)::value><<<grid_of(nE), 256, 0, st>>>(
                d_points, bSplitE_.as<int32_t>(), bSplitCode_.as<int32_t>(), nE,
                bSplitBox_.as<SplitBox>(), bSplitCnt_.as<int32_t>());
            return cudaGetLastError();
        }));
        size_t sb = 0;
        TK(cub::DeviceScan::ExclusiveSum(nullptr, sb, bSplitCnt_.as<int32_t>(), bSplitOff_.as<int32_t>(),
                                         (int)nE, st));
        TK(bTemp_.ensure(sb));
        TK(cub::DeviceScan::ExclusiveSum(bTemp_.p, sb, bSplitCnt_.as<int32_t>(), bSplitOff_.as<int32_t>(),
                                         (int)nE, st));
        int32_t lo_ = 0, lc_ = 0;
        TK(cudaMemcpyAsync(&lo_, bSplitOff_.as<int32_t>() + nE - 1, 4, cudaMemcpyDeviceToHost, st));
        TK(cudaMemcpyAsync(&lc_, bSplitCnt_.as<int32_t>() + nE - 1, 4, cudaMemcpyDeviceToHost, st));
        TK(cudaStreamSynchronize(st));
        const int64_t mo = (int64_t)lo_ + lc_;
        TK(bSplitK_.ensure(4 * (size_t)(mo + 1)));
        TK(bSplitV_.ensure(4 * (size_t)(mo + 1)));
        TK(bSplitK2_.ensure(4 * (size_t)(mo + 1)));
        split_bufs_.emplace_back(new DevBuf());
        DevBuf& vout = *split_bufs_.back();
        TK(vout.ensure(4 * (size_t)(mo + 1)));
        TK(with_dim(dim, [&](auto D) {
            k_split_fill<decltype(D)::value><<<grid_of(nE), 256, 0, st>>>(
                d_points, bSplitE_.as<int32_t>(), bSplitCode_.as<int32_t>(), nE,
                bSplitBox_.as<SplitBox>(), bSplitOff_.as<int32_t>(), bSplitK_.as<uint32_t>(),
                bSplitV_.as<int32_t>());
            return cudaGetLastError();
        }));
        int kbits = 1;
        while ((int64_t(1) << kbits) < 4 * (int64_t)nn) ++kbits;
        sb = 0;
        TK(cub::DeviceRadixSort::SortPairs(nullptr, sb, bSplitK_.as<uint32_t>(), bSplitK2_.as<uint32_t>(),
                                           bSplitV_.as<int32_t>(), vout.as<int32_t>(), (int)mo, 0,
                                           kbits, st));
        TK(bTemp_.ensure(sb));
        TK(cub::DeviceRadixSort::SortPairs(bTemp_.p, sb, bSplitK_.as<uint32_t>(), bSplitK2_.as<uint32_t>(),
                                           bSplitV_.as<int32_t>(), vout.as<int32_t>(), (int)mo, 0,
                                           kbits, st));
        TK(bSplitSeg_.ensure(8 * (size_t)(4 * nn + 1)));
        TK(cudaMemsetAsync(bSplitSeg_.p, 0, 8 * (size_t)(4 * nn), st));
        if (mo > 0) {
            k_seg_bounds<<<grid_of(mo), 256, 0, st>>>(bSplitK2_.as<uint32_t>(), mo, bSplitSeg_.as<int32_t>());
            TK(cudaGetLastError());
        }
        std::vector<int32_t> cseg(8 * (size_t)nn);
        TK(cudaMemcpyAsync(cseg.data(), bSplitSeg_.p, 4 * cseg.size(), cudaMemcpyDeviceToHost, st));
        TK(cudaStreamSynchronize(st));
        // the halves: dropped (< 2 own points), leaves (< cap) or next level
        std::vector<SplitNode> next;
        const int bi = (int)split_bufs_.size() - 1;
        for (int q = 0; q < nn; ++q) {
            for (int sh = 0; sh < 2; ++sh) {
                const int c = 2 * q + sh;
                const int64_t os = cseg[4 * c], oe = cseg[4 * c + 1];
                const int64_t hs = cseg[4 * c + 2], he = cseg[4 * c + 3];
                const int64_t no = oe - os, nh = he - hs;
                if (no <= 1) continue;
                if (nh > 0 && hs != oe) { last_error = "internal: split segments not adjacent"; return 2; }
                const SplitNode& pn = nodes[q];
                const uint64_t path = pn.path | ((uint64_t)sh << (63 - pn.depth));
                if (no < cap) {
                    subleaves.push_back(SubLeaf{pn.root, path, bi, os, no, nh});
                } else {
                    SplitNode ch;
                    ch.box = halves[c];
                    ch.root = pn.root;
                    ch.path = path;
                    ch.depth = pn.depth + 1;
                    ch.src = os;
                    ch.own = no;
                    ch.halo = nh;
                    next.push_back(ch);
                }
            }
        }
        nodes.swap(next);
        src_vals = vout.as<int32_t>();
    }
    std::stable_sort(subleaves.begin(), subleaves.end(), [](const SubLeaf& x, const SubLeaf& y) {
        return x.root != y.root ? x.root < y.root : x.path < y.path;
    });
    size_t nxt = 0;                 // next sub-leaf in pre-order
    std::vector<int64_t> xoffs;     // per sub-leaf (pre-order): offset in the extra points
    int64_t xtotal = 0;
    for (int64_t t = 0; t < ntiles; ++t) {
        int64_t os, oe, hs, he;
        own_of(t, os, oe);
        halo_of(t, hs, he);
        const int64_t no = oe - os, nh = he - hs;
        if (no <= 1) continue;
        if (no < cap) {
            CloudDesc cd;
            std::memset(&cd, 0, sizeof(cd));
            cd.p_off = os;
            cd.n_own = (int32_t)no;
            cd.n_all = (int32_t)(no + nh);
            cd.r1 = r1;
            cd.r2 = r2;
            cl.push_back(cd);
            continue;
        }
        for (; nxt < subleaves.size() && subleaves[nxt].root == t; ++nxt) {
            const SubLeaf& L = subleaves[nxt];
            CloudDesc cd;
            std::memset(&cd, 0, sizeof(cd));
            cd.p_off = m + xtotal;
            cd.n_own = (int32_t)L.own;
            cd.n_all = (int32_t)(L.own + L.halo);
            cd.r1 = r1;
            cd.r2 = r2;
            cl.push_back(cd);
            xoffs.push_back(xtotal);
            xtotal += L.own + L.halo;
        }
    }
    // the sub-leaves' point lists, in pre-order, behind the tiles' lists
    if (xtotal > 0) {
        TK(bExtra_.ensure(4 * (size_t)xtotal));
        for (size_t k = 0; k < subleaves.size(); ++k) {
            const SubLeaf& L = subleaves[k];
            TK(cudaMemcpyAsync(bExtra_.as<int32_t>() + xoffs[k],
                               split_bufs_[L.buf]->as<int32_t>() + L.off,
                               4 * (size_t)(L.own + L.halo), cudaMemcpyDeviceToDevice, st));
        }
    }
    const int64_t total = m + xtotal;
    std::vector<GroupDesc> gr;
    if (local_policy) {
        // RD_LOCAL: every leaf is its own group, decimated on its own with the
        // brute-force semantics (agent_tiled_ridge_detection.cuh:232-331)
        gr.resize(cl.size());
        std::memset(gr.data(), 0, sizeof(GroupDesc) * gr.size());
        for (size_t c = 0; c < cl.size(); ++c) {
            cl[c].group = (int32_t)c;
            gr[c].cloud_begin = (int32_t)c;
            gr[c].n_clouds = 1;
            gr[c].nocopy = 0;
        }
    } else {
        // RD_MIXED: one group of all leaves, global decimateNoCopy
        for (auto& c : cl) c.group = 0;
        gr.resize(1);
        std::memset(gr.data(), 0, sizeof(GroupDesc));
        gr[0].cloud_begin = 0;
        gr[0].n_clouds = (int32_t)cl.size();
        gr[0].nocopy = 1;
    }
    if (cl.empty()) {
        tm_.build_ms = tm_.whole_ms =
            std::chrono::duration<float, std::milli>(clk::now() - t0).count();
        return 0;
    }
    if (int rc = eng_.setup(dim, cl, gr, total)) { last_error = eng_.last_error; return rc; }
    // 7. packed per-leaf evolve points: own then halo, each in input order
    TK(with_dim(dim, [&](auto D) {
        constexpr int DIM = decltype(D)::value;
        k_gather_idx<DIM><<<grid_of(m * DIM), 256, 0, st>>>(d_points, bVals2_.as<int32_t>(), m,
                                                            eng_.points());
        return cudaGetLastError();
    }));
    if (xtotal > 0) {
        const int64_t xm = xtotal;
        TK(with_dim(dim, [&](auto D) {
            constexpr int DIM = decltype(D)::value;
            k_gather_idx<DIM><<<grid_of(xm * DIM), 256, 0, st>>>(d_points, bExtra_.as<int32_t>(), xm,
                                                                 eng_.points() + m * DIM);
            return cudaGetLastError();
        }));
    }
    TK(cudaStreamSynchronize(st));
    const auto t1 = clk::now();
    tm_.build_ms = std::chrono::duration<float, std::milli>(t1 - t0).count();

    // 8. choose / evolve / global decimate on the device
    int rc = eng_.run(st, use_graph);
    if (rc && rc != 4) { last_error = eng_.last_error; return rc; }
    // 9. collect in leaf pre-order
    const auto& nsv = eng_.ns();
    const auto& ecl = eng_.clouds();
    std::vector<int64_t> tab(3 * ecl.size());
    int64_t outoff = 0;
    leaf_ns_.assign(nsv.begin(), nsv.end());
    for (size_t l = 0; l < ecl.size(); ++l) {
        tab[3 * l] = ecl[l].s_off * dim;
        tab[3 * l + 1] = (int64_t)nsv[l] * dim;
        tab[3 * l + 2] = outoff;
        outoff += (int64_t)nsv[l] * dim;
    }
    ns_ = outoff / dim;
    TK(bOut_.ensure(sizeof(float) * (size_t)(outoff + 1)));
    TK(bTab_.ensure(sizeof(int64_t) * tab.size()));
    TK(cudaMemcpyAsync(bTab_.p, tab.data(), sizeof(int64_t) * tab.size(), cudaMemcpyHostToDevice, st));
    dim3 grid(8, (unsigned)std::min<size_t>(ecl.size(), 65535));
    k_concat<<<grid, 256, 0, st>>>(eng_.chosen(), bTab_.as<int64_t>(), (int)ecl.size(), bOut_.as<float>());
    TK(cudaGetLastError());
    TK(cudaStreamSynchronize(st));
    const auto t2 = clk::now();
    tm_.rd_ms = std::chrono::duration<float, std::milli>(t2 - t1).count();
    tm_.whole_ms = std::chrono::duration<float, std::milli>(t2 - t0).count();
    if (rc) last_error = eng_.last_error;
    return rc;
}

}  // namespace rdb
