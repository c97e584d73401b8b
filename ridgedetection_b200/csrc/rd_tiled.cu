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

constexpr int MAXD = 3;

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

bool is_inside(const HBox& b, const float* p, int dim)
{
    for (int d = 0; d < dim; ++d)
        if (p[d] < b.mn[d] || p[d] >= b.mx[d]) return false;
    return true;
}

bool is_nearby(const HBox& b, const float* p, float r, int dim)
{
    for (int d = 0; d < dim; ++d) {
        const volatile float emin = b.mn[d] - r;
        const volatile float emax = b.mx[d] + r;
        if (p[d] < emin || p[d] >= emax) return false;
    }
    return !is_inside(b, p, dim);
}

struct HostLeaf {
    std::vector<int32_t> own, halo;
};

// grouped_tile_tree.inl:247-330: half-split along dimension level % dim over
// the parent's own points, then its halo; drop sub-tiles with < 2 own points;
// recurse while own points >= cap.
bool split_tile(const HBox& parent, const std::vector<int32_t>& own,
                const std::vector<int32_t>& halo, int level, int64_t cap, float r,
                const float* P, int dim, std::vector<HostLeaf>& out)
{
    if (level > 64) return false;
    const int sd = level % dim;
    HBox sub[2];
    for (int s = 0; s < 2; ++s) {
        for (int d = 0; d < dim; ++d) {
            if (d == sd) tile_bounds(parent, d, s, 2, sub[s].mn[d], sub[s].mx[d]);
            else tile_bounds(parent, d, 0, 1, sub[s].mn[d], sub[s].mx[d]);
        }
        calc_dist(sub[s], dim);
    }
    std::vector<int32_t> so[2], sh[2];
    for (int32_t i : own) {
        const float* p = P + (int64_t)i * dim;
        for (int s = 0; s < 2; ++s)
            if (is_nearby(sub[s], p, r, dim)) sh[s].push_back(i);
        for (int s = 0; s < 2; ++s)
            if (is_inside(sub[s], p, dim)) { so[s].push_back(i); break; }
    }
    for (int32_t i : halo) {
        const float* p = P + (int64_t)i * dim;
        for (int s = 0; s < 2; ++s)
            if (is_nearby(sub[s], p, r, dim)) sh[s].push_back(i);
    }
    for (int s = 0; s < 2; ++s) {
        if (so[s].size() <= 1) continue;
        if ((int64_t)so[s].size() < cap) {
            out.push_back(HostLeaf{std::move(so[s]), std::move(sh[s])});
        } else if (!split_tile(sub[s], so[s], sh[s], level + 1, cap, r, P, dim, out)) {
            return false;
        }
    }
    return true;
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
    if (dim != 2 && dim != 3) { last_error = "dim must be 2 or 3"; return 6; }
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
    if (dim == 2) k_bbox<2><<<grid_of(n), 256, 0, st>>>(d_points, n, bBox_.as<int>());
    else k_bbox<3><<<grid_of(n), 256, 0, st>>>(d_points, n, bBox_.as<int>());
    TK(cudaGetLastError());
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
    if (dim == 2) k_emit_count<2><<<grid_of(n), 256, 0, st>>>(d_points, n, gd, tmin, tmax, bCnt_.as<int32_t>());
    else k_emit_count<3><<<grid_of(n), 256, 0, st>>>(d_points, n, gd, tmin, tmax, bCnt_.as<int32_t>());
    TK(cudaGetLastError());
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
    if (dim == 2)
        k_emit_fill<2><<<grid_of(n), 256, 0, st>>>(d_points, n, gd, tmin, tmax, bOff_.as<int32_t>(),
                                                  bKeys_.as<uint32_t>(), bVals_.as<int32_t>());
    else
        k_emit_fill<3><<<grid_of(n), 256, 0, st>>>(d_points, n, gd, tmin, tmax, bOff_.as<int32_t>(),
                                                  bKeys_.as<uint32_t>(), bVals_.as<int32_t>());
    TK(cudaGetLastError());
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

    // 6. leaves in pre-order; oversize tiles are split on the host
    std::vector<CloudDesc> cl;
    std::vector<HostLeaf> extra;
    std::vector<int64_t> extra_at;  // leaf index of each extra leaf
    std::vector<float> hP;
    auto own_of = [&](int64_t t, int64_t& s, int64_t& e) { s = seg[4 * t]; e = seg[4 * t + 1]; };
    auto halo_of = [&](int64_t t, int64_t& s, int64_t& e) { s = seg[4 * t + 2]; e = seg[4 * t + 3]; };
    for (int64_t t = 0; t < ntiles; ++t) {
        int64_t os, oe, hs, he;
        own_of(t, os, oe);
        halo_of(t, hs, he);
        const int64_t no = oe - os, nh = he - hs;
        if (no <= 1) continue;
        if (no < cap) {
            if (nh > 0 && hs != oe) { last_error = "internal: tile segments not adjacent"; return 2; }
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
        if (hP.empty()) {
            hP.resize((size_t)n * dim);
            TK(cudaMemcpyAsync(hP.data(), d_points, sizeof(float) * n * dim, cudaMemcpyDeviceToHost, st));
            TK(cudaStreamSynchronize(st));
        }
        std::vector<int32_t> own((size_t)no), halo((size_t)nh);
        TK(cudaMemcpyAsync(own.data(), bVals2_.as<int32_t>() + os, 4 * no, cudaMemcpyDeviceToHost, st));
        if (nh) TK(cudaMemcpyAsync(halo.data(), bVals2_.as<int32_t>() + hs, 4 * nh, cudaMemcpyDeviceToHost, st));
        TK(cudaStreamSynchronize(st));
        HBox tb_;
        int64_t rem = t;
        for (int d = 0; d < dim; ++d) {
            const int c = (int)(rem % tpd[d]);
            rem /= tpd[d];
            tb_.mn[d] = hb[gd.off[d] + c];
            tb_.mx[d] = hb[tot + gd.off[d] + c];
        }
        calc_dist(tb_, dim);
        std::vector<HostLeaf> sub;
        if (!split_tile(tb_, own, halo, 1, cap, r1, hP.data(), dim, sub)) {
            last_error = "tile subdivision did not terminate (duplicate points above capacity)";
            return 1;
        }
        for (auto& L : sub) {
            CloudDesc cd;
            std::memset(&cd, 0, sizeof(cd));
            cd.n_own = (int32_t)L.own.size();
            cd.n_all = (int32_t)(L.own.size() + L.halo.size());
            cd.r1 = r1;
            cd.r2 = r2;
            cd.p_off = -1;  // filled below
            extra_at.push_back((int64_t)cl.size());
            cl.push_back(cd);
            extra.push_back(std::move(L));
        }
    }
    std::vector<int32_t> xidx;
    for (size_t k = 0; k < extra.size(); ++k) {
        cl[extra_at[k]].p_off = m + (int64_t)xidx.size();
        xidx.insert(xidx.end(), extra[k].own.begin(), extra[k].own.end());
        xidx.insert(xidx.end(), extra[k].halo.begin(), extra[k].halo.end());
    }
    const int64_t total = m + (int64_t)xidx.size();
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
    if (dim == 2) k_gather_idx<2><<<grid_of(m * 2), 256, 0, st>>>(d_points, bVals2_.as<int32_t>(), m, eng_.points());
    else k_gather_idx<3><<<grid_of(m * 3), 256, 0, st>>>(d_points, bVals2_.as<int32_t>(), m, eng_.points());
    TK(cudaGetLastError());
    if (!xidx.empty()) {
        TK(bExtra_.ensure(4 * xidx.size()));
        TK(cudaMemcpyAsync(bExtra_.p, xidx.data(), 4 * xidx.size(), cudaMemcpyHostToDevice, st));
        const int64_t xm = (int64_t)xidx.size();
        if (dim == 2) k_gather_idx<2><<<grid_of(xm * 2), 256, 0, st>>>(d_points, bExtra_.as<int32_t>(), xm, eng_.points() + m * 2);
        else k_gather_idx<3><<<grid_of(xm * 3), 256, 0, st>>>(d_points, bExtra_.as<int32_t>(), xm, eng_.points() + m * 3);
        TK(cudaGetLastError());
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
