/*
 * rd_oracle.c -- CPU restatement of the reference's choose / evolve / decimate
 * path (brute-force and extended-tile tiled variants), in plain C.
 *
 * TEST INFRASTRUCTURE ONLY: loaded by tests/, __graft_entry__.smoke() and the
 * CPU-baseline leg of bench.py as the checker.  The product never links it.
 *
 * Parity pin: tests/test_oracle.py compares every entry point bit for bit with
 * the reference's own code compiled from its sources (oracle/ref_shim.cpp) on
 * the seeded fixtures in tests/golden/.  Build with -ffp-contract=off so that
 * no multiply-add is fused: the reference's x86-64 build rounds every product
 * and every sum separately.
 *
 * Reference file:line citations are paths inside ridge_detection/ of
 * aosewski/RidgeDetection.
 */
#include "rd_oracle.h"

#include <float.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

/* rd/cpu/brute_force/rd_inner.hpp:42-49 (squareEuclideanDistance):
 * acc starts at 0, t = a - b, acc += t*t in dimension order. */
static inline float sqdist(const float* a, const float* b, int dim)
{
    float acc = 0.0f;
    for (int d = 0; d < dim; ++d) {
        float t = a[d] - b[d];
        acc += t * t;
    }
    return acc;
}

/* rd/cpu/brute_force/choose.hpp:37-70: first point chosen; point k is chosen iff
 * no already-chosen point lies at squared distance <= r1*r1 (rd_inner.hpp:67-86,
 * threshold 1).  Chosen points are copied to S in visiting order. */
int64_t rdo_choose(const float* P, int64_t np, int dim, float r1, float* S)
{
    if (np <= 0) return 0;
    const float rsq = r1 * r1;
    int64_t ns = 0;
    memcpy(S, P, sizeof(float) * (size_t)dim);
    ns = 1;
    for (int64_t i = 1; i < np; ++i) {
        const float* p = P + i * dim;
        int hit = 0;
        for (int64_t k = 0; k < ns; ++k) {
            if (sqdist(p, S + k * dim, dim) <= rsq) { hit = 1; break; }
        }
        if (!hit) {
            memcpy(S + ns * dim, p, sizeof(float) * (size_t)dim);
            ++ns;
        }
    }
    return ns;
}

/* rd/cpu/brute_force/evolve.hpp:43-66 (calculateClosestSphereCenter, argmin part):
 * key[i] = index of the nearest chosen point (strict '<', so the lowest index
 * wins ties, minimum starts at FLT_MAX) if that distance is <= r1*r1, else -1.
 * The distance there is computed as (S - P), which squares to the same value. */
void rdo_assign(const float* P, int64_t np, const float* S, int64_t ns, int dim,
                float r1, int32_t* key)
{
    const float rsq = r1 * r1;
    for (int64_t n = 0; n < np; ++n) {
        const float* p = P + n * dim;
        float best = FLT_MAX;
        int32_t bi = -1;
        for (int64_t k = 0; k < ns; ++k) {
            float acc = 0.0f;
            for (int d = 0; d < dim; ++d) {
                float t = S[k * dim + d] - p[d];
                acc += t * t;
            }
            if (acc < best) { best = acc; bi = (int32_t)k; }
        }
        key[n] = (best <= rsq) ? bi : -1;
    }
}

/* rd/cpu/brute_force/evolve.hpp:66-75: counts and FP32 coordinate sums,
 * accumulated in cloud-point index order starting from zero. */
void rdo_accumulate(const float* P, int64_t np, const int32_t* key, int64_t ns, int dim,
                    float* sums, int32_t* cnt)
{
    memset(sums, 0, sizeof(float) * (size_t)(ns * dim));
    memset(cnt, 0, sizeof(int32_t) * (size_t)ns);
    for (int64_t n = 0; n < np; ++n) {
        int32_t k = key[n];
        if (k < 0) continue;
        cnt[k]++;
        for (int d = 0; d < dim; ++d) sums[(int64_t)k * dim + d] += P[n * dim + d];
    }
}

/* rd/cpu/brute_force/evolve.hpp:130-179 (shiftTowardMassCenter): per coordinate,
 * mc = sum/cnt (skipped when cnt == 0); the coordinate moves to mc and the
 * continue flag is raised iff |mc - c| > 2.f*|mc|*cnt*FLT_EPSILON, evaluated
 * left to right in float. */
int rdo_shift(float* S, const float* sums, const int32_t* cnt, int64_t ns, int dim)
{
    int cont = 0;
    for (int64_t k = 0; k < ns; ++k) {
        if (cnt[k] == 0) continue;
        const float fc = (float)cnt[k];
        for (int d = 0; d < dim; ++d) {
            float mc = sums[k * dim + d] / fc;
            float thr = 2.0f * fabsf(mc);
            thr = thr * fc;
            thr = thr * FLT_EPSILON;
            if (fabsf(mc - S[k * dim + d]) > thr) {
                cont = 1;
                S[k * dim + d] = mc;
            }
        }
    }
    return cont;
}

int rdo_evolve_pass(const float* P, int64_t np, float* S, int64_t ns, int dim, float r1,
                    float* sums, int32_t* cnt, int32_t* key)
{
    rdo_assign(P, np, S, ns, dim, r1, key);
    rdo_accumulate(P, np, key, ns, dim, sums, cnt);
    return rdo_shift(S, sums, cnt, ns, dim);
}

/* rd/cpu/brute_force/evolve.hpp:293-342 (evolve): passes until no coordinate
 * moved.  Returns the number of passes (or -1 if max_passes > 0 ran out). */
int64_t rdo_evolve(const float* P, int64_t np, float* S, int64_t ns, int dim, float r1,
                   int64_t max_passes, double* pairs)
{
    float* sums = (float*)malloc(sizeof(float) * (size_t)(ns * dim + 1));
    int32_t* cnt = (int32_t*)malloc(sizeof(int32_t) * (size_t)(ns + 1));
    int32_t* key = (int32_t*)malloc(sizeof(int32_t) * (size_t)(np + 1));
    int64_t passes = 0;
    int cont = 1;
    while (cont) {
        if (max_passes > 0 && passes >= max_passes) { passes = -1; break; }
        cont = rdo_evolve_pass(P, np, S, ns, dim, r1, sums, cnt, key);
        ++passes;
        if (pairs) *pairs += (double)np * (double)ns;
    }
    free(sums); free(cnt); free(key);
    return passes;
}

/* Neighbour count of S[i] among alive points (self included), as
 * countNeighbouringPoints over a list (rd_inner.hpp:113-133) without the
 * early exit, which only shortens the scan. */
static int64_t count_alive(const float* S, const unsigned char* alive, int64_t ns, int dim,
                           int64_t i, float rsq)
{
    int64_t c = 0;
    for (int64_t j = 0; j < ns; ++j)
        if (alive[j] && sqdist(S + i * dim, S + j * dim, dim) <= rsq) ++c;
    return c;
}

/* rd/cpu/brute_force/decimate.hpp:41-81 (decimate): in list order, remove a
 * point if it has >= 4 alive points within r2 (self included) or < 3 within
 * 2*r2 (radius^2 = 4.f*r2^2); removal is immediate.  Passes repeat while a pass
 * removed something and more than 3 remain; a pass stops as soon as fewer than
 * 3 remain.  Survivors are compacted to the front of S in order. */
int64_t rdo_decimate(float* S, int64_t ns, int dim, float r2)
{
    const float rsq = r2 * r2;
    const float rsq4 = 4.0f * rsq;
    unsigned char* alive = (unsigned char*)malloc((size_t)ns + 1);
    memset(alive, 1, (size_t)ns + 1);
    int64_t cnt = ns, left = 0;
    while (left != cnt && cnt > 3) {
        left = cnt;
        for (int64_t i = 0; i < ns; ++i) {
            if (!alive[i]) continue;
            if (count_alive(S, alive, ns, dim, i, rsq) >= 4 ||
                count_alive(S, alive, ns, dim, i, rsq4) < 3) {
                alive[i] = 0;
                --cnt;
                if (cnt < 3) break;
            }
        }
    }
    int64_t w = 0;
    for (int64_t i = 0; i < ns; ++i)
        if (alive[i]) {
            if (w != i) memmove(S + w * dim, S + i * dim, sizeof(float) * (size_t)dim);
            ++w;
        }
    free(alive);
    return w;
}

/* rd/cpu/brute_force/decimate.hpp:85-127 (decimateNoCopy) over consecutive
 * segments of S (one per tile, in leaf order).  Same removal test as above,
 * but a point that qualifies is kept when removing it would leave fewer than 3
 * (csCnt - 1 < 3) and the scan goes on.  std::list::remove_if unlinks each
 * element as soon as the predicate is true, so later counts exclude it.
 * Survivors are compacted in order; seg_cnt is updated. */
int64_t rdo_decimate_seg(float* S, int64_t nseg, int64_t* seg_cnt, int dim, float r2)
{
    const float rsq = r2 * r2;
    const float rsq4 = 4.0f * rsq;
    int64_t ns = 0;
    for (int64_t s = 0; s < nseg; ++s) ns += seg_cnt[s];
    unsigned char* alive = (unsigned char*)malloc((size_t)ns + 1);
    memset(alive, 1, (size_t)ns + 1);
    int64_t cnt = ns, left = 0;
    while (left != cnt && cnt > 3) {
        left = cnt;
        for (int64_t i = 0; i < ns; ++i) {
            if (!alive[i]) continue;
            if (count_alive(S, alive, ns, dim, i, rsq) >= 4 ||
                count_alive(S, alive, ns, dim, i, rsq4) < 3) {
                if (cnt - 1 < 3) continue;
                alive[i] = 0;
                --cnt;
            }
        }
    }
    int64_t w = 0, base = 0;
    for (int64_t s = 0; s < nseg; ++s) {
        int64_t kept = 0;
        for (int64_t i = base; i < base + seg_cnt[s]; ++i)
            if (alive[i]) {
                if (w != i) memmove(S + w * dim, S + i * dim, sizeof(float) * (size_t)dim);
                ++w; ++kept;
            }
        base += seg_cnt[s];
        seg_cnt[s] = kept;
    }
    free(alive);
    return w;
}

/* rd/cpu/brute_force/ridge_detection.inl:68-146 (ridgeDetection, serial):
 * choose, then {evolve; decimate} until the chosen count stops changing. */
int64_t rdo_ridge_bf(const float* P, int64_t np, int dim, float r1, float r2, float* S,
                     rdo_stats* st)
{
    int64_t ns = rdo_choose(P, np, dim, r1, S);
    if (st) { memset(st, 0, sizeof(*st)); st->ns_choose = ns; }
    int64_t old = 0;
    while (old != ns) {
        old = ns;
        double pairs = 0;
        int64_t passes = rdo_evolve(P, np, S, ns, dim, r1, 0, &pairs);
        ns = rdo_decimate(S, ns, dim, r2);
        if (st) { st->outer_iters++; st->evolve_passes += passes; st->pairs += pairs; }
    }
    return ns;
}

/* ------------------------------------------------------------------------- */
/* Tiled variant: rd/cpu/tiled/rd_tiled.hpp:1217-1374 (EXT_TILE_TREE_MIXED_RD)
 * over the extended-tile tree of rd/cpu/tiled/grouped_tile_tree.inl.          */
/* ------------------------------------------------------------------------- */

typedef struct { int64_t* v; int64_t n, cap; } ivec;

static void iv_push(ivec* a, int64_t x)
{
    if (a->n == a->cap) {
        a->cap = a->cap ? a->cap * 2 : 16;
        a->v = (int64_t*)realloc(a->v, sizeof(int64_t) * (size_t)a->cap);
    }
    a->v[a->n++] = x;
}

typedef struct otile {
    float min[8], max[8], dist[8];
    ivec samples;    /* cloud indices of own points, in visiting order     */
    ivec halo;       /* cloud indices of the r1-extended neighbourhood     */
} otile;

typedef struct { otile** v; int64_t n, cap; } tvec;

static void tv_push(tvec* a, otile* t)
{
    if (a->n == a->cap) {
        a->cap = a->cap ? a->cap * 2 : 16;
        a->v = (otile**)realloc(a->v, sizeof(otile*) * (size_t)a->cap);
    }
    a->v[a->n++] = t;
}

/* rd/utils/bounding_box.hpp:210-227 (calcDistances) */
static void calc_dist(otile* t, int dim)
{
    for (int d = 0; d < dim; ++d) {
        float x = fabsf(t->max[d] - t->min[d]);
        t->dist[d] = (x <= FLT_EPSILON) ? 0.0f : x;
    }
}

/* rd/utils/bounding_box.hpp:335-344: min <= x < max in every dimension */
static int is_inside(const otile* t, const float* p, int dim)
{
    for (int d = 0; d < dim; ++d)
        if (p[d] < t->min[d] || p[d] >= t->max[d]) return 0;
    return 1;
}

/* rd/utils/bounding_box.hpp:360-375: inside the box grown by r, not inside */
static int is_nearby(const otile* t, const float* p, float r, int dim)
{
    for (int d = 0; d < dim; ++d)
        if (p[d] < t->min[d] - r || p[d] >= t->max[d] + r) return 0;
    return !is_inside(t, p, dim);
}

/* grouped_tile_tree.inl:147-213 (allocTiles): tile coordinates advance with
 * dimension 0 fastest; min = bmin + c*step, max = bmin + (c+1)*step, and the
 * last tile of each dimension takes the parent's max. */
static void alloc_tiles(const otile* box, int dim, const int64_t* cnt, tvec* out)
{
    float step[8];
    int64_t n = 1;
    for (int d = 0; d < dim; ++d) { step[d] = box->dist[d] / (float)cnt[d]; n *= cnt[d]; }
    int64_t c[8];
    for (int64_t i = 0; i < n; ++i) {
        int64_t r = i;
        otile* t = (otile*)calloc(1, sizeof(otile));
        for (int d = 0; d < dim; ++d) { c[d] = r % cnt[d]; r /= cnt[d]; }
        for (int d = 0; d < dim; ++d) {
            float lo = (float)c[d] * step[d];
            float hi = (float)(c[d] + 1) * step[d];
            t->min[d] = box->min[d] + lo;
            t->max[d] = box->min[d] + hi;
            if (c[d] == cnt[d] - 1) t->max[d] = box->max[d];
        }
        calc_dist(t, dim);
        tv_push(out, t);
    }
}

/* grouped_tile_tree.inl:445-511 (EXTENDED_TILE partitionSamples) for one
 * source list: every tile whose extended box holds the point (and not the
 * tile itself) appends it to its halo; for the own-sample list (is_own) the
 * first tile holding it appends it to its samples.  The point loop is the
 * outer loop, so every list keeps the source order. */
static void partition(const float* P, int dim, const ivec* src, int is_own, float r,
                      tvec* tiles)
{
    for (int64_t a = 0; a < src->n; ++a) {
        const int64_t i = src->v[a];
        const float* p = P + i * dim;
        for (int64_t t = 0; t < tiles->n; ++t)
            if (is_nearby(tiles->v[t], p, r, dim)) iv_push(&tiles->v[t]->halo, i);
        if (is_own)
            for (int64_t t = 0; t < tiles->n; ++t)
                if (is_inside(tiles->v[t], p, dim)) { iv_push(&tiles->v[t]->samples, i); break; }
    }
}

static void free_tile(otile* t)
{
    free(t->samples.v);
    free(t->halo.v);
    free(t);
}

/* grouped_tile_tree.inl:216-244: drop tiles with 0 or 1 own points. */
static void reduce_tiles(tvec* tiles)
{
    int64_t w = 0;
    for (int64_t t = 0; t < tiles->n; ++t) {
        if (tiles->v[t]->samples.n <= 1) free_tile(tiles->v[t]);
        else tiles->v[w++] = tiles->v[t];
    }
    tiles->n = w;
}

typedef struct {
    const float* P;
    int dim;
    float r1;
    int64_t cap;
    tvec leaves;     /* preorder */
    int err;
} tree_ctx;

/* grouped_tile_tree.inl:247-330 (addNode / subdivideTile): a tile with
 * fewer than cap own points is a leaf; otherwise it is half-split along
 * dimension (level % dim) over its own points then its halo, recursively. */
static void add_node(tree_ctx* cx, otile* t, int level)
{
    if (t->samples.n < cx->cap) { tv_push(&cx->leaves, t); return; }
    if (level > 64) { cx->err = 1; free_tile(t); return; }
    int64_t cnt[8];
    for (int d = 0; d < cx->dim; ++d) cnt[d] = 1;
    cnt[level % cx->dim] = 2;
    tvec sub = {0};
    alloc_tiles(t, cx->dim, cnt, &sub);
    partition(cx->P, cx->dim, &t->samples, 1, cx->r1, &sub);
    partition(cx->P, cx->dim, &t->halo, 0, cx->r1, &sub);
    reduce_tiles(&sub);
    free_tile(t);
    for (int64_t s = 0; s < sub.n; ++s) add_node(cx, sub.v[s], level + 1);
    free(sub.v);
}

/* rd_tiled.hpp:1217-1374.  S receives the final chosen points of all leaves in
 * preorder; n_leaves (optional) the number of leaves. */
int64_t rdo_ridge_tiled(const float* P, int64_t np, int dim, float r1, float r2,
                        int64_t max_tile_capacity, const int64_t* tiles_per_dim,
                        float* S, int64_t* n_leaves, rdo_stats* st)
{
    return rdo_ridge_tiled_policy(P, np, dim, r1, r2, max_tile_capacity, tiles_per_dim, 0, S,
                                  n_leaves, st);
}

/* local = 0: EXT_TILE_TREE_MIXED_RD (rd_tiled.hpp:1217-1374), local evolve and
 * a global decimateNoCopy.  local = 1: the RD_LOCAL policy of the GPU
 * reference (agent_tiled_ridge_detection.cuh:232-331 over the same extended
 * tiles; dispatch_ridge_detection.cuh doApproximate): every leaf on its own,
 * choose over its own points, then (evolve over own + halo points; brute-force
 * decimate) until its count stops changing; results in leaf preorder (the
 * reference appends leaves in completion order). */
int64_t rdo_ridge_tiled_policy(const float* P, int64_t np, int dim, float r1, float r2,
                               int64_t max_tile_capacity, const int64_t* tiles_per_dim,
                               int local, float* S, int64_t* n_leaves, rdo_stats* st)
{
    if (st) memset(st, 0, sizeof(*st));
    if (np <= 0 || dim < 1 || dim > 8) return 0;
    /* rd/utils/bounding_box.hpp:126-197 (findBounds, serial) */
    otile g;
    memset(&g, 0, sizeof(g));
    for (int d = 0; d < dim; ++d) { g.min[d] = FLT_MAX; g.max[d] = -FLT_MAX; }
    for (int64_t i = 0; i < np; ++i)
        for (int d = 0; d < dim; ++d) {
            float v = P[i * dim + d];
            g.min[d] = (v < g.min[d]) ? v : g.min[d];
            g.max[d] = (v > g.max[d]) ? v : g.max[d];
        }
    calc_dist(&g, dim);

    tree_ctx cx;
    memset(&cx, 0, sizeof(cx));
    cx.P = P; cx.dim = dim; cx.r1 = r1; cx.cap = max_tile_capacity;
    tvec roots = {0};
    alloc_tiles(&g, dim, tiles_per_dim, &roots);
    ivec all = {0};
    for (int64_t i = 0; i < np; ++i) iv_push(&all, i);
    partition(P, dim, &all, 1, r1, &roots);
    free(all.v);
    reduce_tiles(&roots);
    for (int64_t t = 0; t < roots.n; ++t) add_node(&cx, roots.v[t], 1);
    free(roots.v);
    if (n_leaves) *n_leaves = cx.leaves.n;

    const int64_t nl = cx.leaves.n;
    /* per-leaf gathered coordinates: own points then halo (tile.hpp:167-176) */
    float** pts = (float**)calloc((size_t)nl + 1, sizeof(float*));
    int64_t* npts = (int64_t*)calloc((size_t)nl + 1, sizeof(int64_t));
    int64_t* nown = (int64_t*)calloc((size_t)nl + 1, sizeof(int64_t));
    float** chosen = (float**)calloc((size_t)nl + 1, sizeof(float*));
    int64_t* nch = (int64_t*)calloc((size_t)nl + 1, sizeof(int64_t));
    int64_t ns = 0;
    for (int64_t l = 0; l < nl; ++l) {
        otile* t = cx.leaves.v[l];
        nown[l] = t->samples.n;
        npts[l] = t->samples.n + t->halo.n;
        pts[l] = (float*)malloc(sizeof(float) * (size_t)(npts[l] * dim + 1));
        for (int64_t a = 0; a < t->samples.n; ++a)
            memcpy(pts[l] + a * dim, P + t->samples.v[a] * dim, sizeof(float) * (size_t)dim);
        for (int64_t a = 0; a < t->halo.n; ++a)
            memcpy(pts[l] + (t->samples.n + a) * dim, P + t->halo.v[a] * dim,
                   sizeof(float) * (size_t)dim);
        /* choose over the tile's own points (rd_tiled.hpp:1255-1263) */
        chosen[l] = (float*)malloc(sizeof(float) * (size_t)(nown[l] * dim + 1));
        nch[l] = rdo_choose(pts[l], nown[l], dim, r1, chosen[l]);
        ns += nch[l];
    }
    if (st) st->ns_choose = ns;

    float* gS = (float*)malloc(sizeof(float) * (size_t)(ns * dim + 1));
    int64_t old = 0;
    if (local) {
        for (int64_t l = 0; l < nl; ++l) {
            int64_t oldc = 0;
            while (oldc != nch[l]) {
                oldc = nch[l];
                double pairs = 0;
                int64_t passes = rdo_evolve(pts[l], npts[l], chosen[l], nch[l], dim, r1, 0, &pairs);
                if (st) { st->evolve_passes += passes; st->pairs += pairs; st->outer_iters++; }
                nch[l] = rdo_decimate(chosen[l], nch[l], dim, r2);
            }
        }
        old = ns;  /* skips the global loop */
    }
    while (old != ns) {
        old = ns;
        /* evolve each leaf against its own chosen set (rd_tiled.hpp:1322-1332) */
        for (int64_t l = 0; l < nl; ++l) {
            double pairs = 0;
            int64_t passes = rdo_evolve(pts[l], npts[l], chosen[l], nch[l], dim, r1, 0, &pairs);
            if (st) { st->evolve_passes += passes; st->pairs += pairs; }
        }
        /* global decimateNoCopy over all leaves in leaf order (:1335) */
        int64_t w = 0;
        for (int64_t l = 0; l < nl; ++l) {
            memcpy(gS + w * dim, chosen[l], sizeof(float) * (size_t)(nch[l] * dim));
            w += nch[l];
        }
        ns = rdo_decimate_seg(gS, nl, nch, dim, r2);
        w = 0;
        for (int64_t l = 0; l < nl; ++l) {
            memcpy(chosen[l], gS + w * dim, sizeof(float) * (size_t)(nch[l] * dim));
            w += nch[l];
        }
        if (st) st->outer_iters++;
    }
    /* collect in leaf preorder (:1362-1374) */
    int64_t w = 0;
    for (int64_t l = 0; l < nl; ++l) {
        memcpy(S + w * dim, chosen[l], sizeof(float) * (size_t)(nch[l] * dim));
        w += nch[l];
    }
    for (int64_t l = 0; l < nl; ++l) {
        free(pts[l]); free(chosen[l]); free_tile(cx.leaves.v[l]);
    }
    free(pts); free(npts); free(nown); free(chosen); free(nch); free(gS);
    free(cx.leaves.v);
    return cx.err ? -1 : w;
}

/* rd/utils/assessment_quality.hpp:91-111: symmetric Hausdorff distance, max of
 * the two directed max-min distances, here in double. */
double rdo_hausdorff(const float* A, int64_t na, const float* B, int64_t nb, int dim)
{
    if (na <= 0 || nb <= 0) return -1.0;
    double h = 0.0;
    for (int pass = 0; pass < 2; ++pass) {
        const float* X = pass ? B : A;
        const float* Y = pass ? A : B;
        int64_t nx = pass ? nb : na, ny = pass ? na : nb;
        for (int64_t i = 0; i < nx; ++i) {
            double best = INFINITY;
            for (int64_t j = 0; j < ny; ++j) {
                double acc = 0;
                for (int d = 0; d < dim; ++d) {
                    double t = (double)X[i * dim + d] - (double)Y[j * dim + d];
                    acc += t * t;
                }
                if (acc < best) best = acc;
            }
            if (best > h) h = best;
        }
    }
    return sqrt(h);
}

/* ------------------------------------------------------------------------- */
/* Evolve adjoint (no reference counterpart).
 * Forward, `iters` passes: A^t = assignment of P to S^{t-1} computed exactly as
 * rdo_assign (FP32); S^t_k = mean of {P_i : i in A^t_k} when |A^t_k| > 0, else
 * S^{t-1}_k.  The mean is the FP32 sum in index order divided by the count, as
 * the evolve pass computes it, but with no movement threshold.  S^0 is given
 * (copies of chosen cloud points).  Loss L = sum_k <W_k, S^iters_k>.
 * Reverse (FP64, assignments frozen): g = W; for t = iters..1, each cluster
 * with |A^t_k| > 0 sends g_k/|A^t_k| to every member and resets g_k = 0;
 * empty clusters pass g_k to S^{t-1}.  What is left in g is dL/dS^0.
 * grad_P (np*dim doubles) receives the cloud-point part; grad_S0 (optional,
 * ns*dim doubles) receives dL/dS^0, which a caller adds to the cloud points
 * S^0 was copied from.  S_final (optional) gets S^iters.  Returns 0 on success. */
int rdo_evolve_adjoint(const float* P, int64_t np, const float* S0, int64_t ns, int dim,
                       float r1, int iters, const double* W, double* grad_P,
                       double* grad_S0, float* S_final)
{
    int32_t* keys = (int32_t*)malloc(sizeof(int32_t) * (size_t)(np * (int64_t)iters + 1));
    int32_t* cnt = (int32_t*)malloc(sizeof(int32_t) * (size_t)(ns * (int64_t)iters + 1));
    float* S = (float*)malloc(sizeof(float) * (size_t)(ns * dim + 1));
    float* sums = (float*)malloc(sizeof(float) * (size_t)(ns * dim + 1));
    double* g = (double*)malloc(sizeof(double) * (size_t)(ns * dim + 1));
    if (!keys || !cnt || !S || !sums || !g) return 1;
    memcpy(S, S0, sizeof(float) * (size_t)(ns * dim));
    for (int t = 0; t < iters; ++t) {
        int32_t* kt = keys + (int64_t)t * np;
        int32_t* ct = cnt + (int64_t)t * ns;
        rdo_assign(P, np, S, ns, dim, r1, kt);
        rdo_accumulate(P, np, kt, ns, dim, sums, ct);
        for (int64_t k = 0; k < ns; ++k) {
            if (ct[k] == 0) continue;
            for (int d = 0; d < dim; ++d) S[k * dim + d] = sums[k * dim + d] / (float)ct[k];
        }
    }
    if (S_final) memcpy(S_final, S, sizeof(float) * (size_t)(ns * dim));
    memcpy(g, W, sizeof(double) * (size_t)(ns * dim));
    memset(grad_P, 0, sizeof(double) * (size_t)(np * dim));
    for (int t = iters - 1; t >= 0; --t) {
        const int32_t* kt = keys + (int64_t)t * np;
        const int32_t* ct = cnt + (int64_t)t * ns;
        for (int64_t i = 0; i < np; ++i) {
            int32_t k = kt[i];
            if (k < 0) continue;
            for (int d = 0; d < dim; ++d)
                grad_P[i * dim + d] += g[(int64_t)k * dim + d] / (double)ct[k];
        }
        for (int64_t k = 0; k < ns; ++k)
            if (ct[k] > 0)
                for (int d = 0; d < dim; ++d) g[k * dim + d] = 0.0;
    }
    if (grad_S0) memcpy(grad_S0, g, sizeof(double) * (size_t)(ns * dim));
    free(keys); free(cnt); free(S); free(sums); free(g);
    return 0;
}

/* ------------------------------------------------------------------------- */
/* rd/cpu/brute_force/order.hpp:45-141 (orderSamples) with the condition of   */
/* ridge_detection.inl:148-168 (squared distance <= r2*r2): greedy chains.     */
/* Every remaining point, in index order, seeds a chain; the chain then takes  */
/* the first later remaining point within r2 of its front (tested first) or of */
/* its back, again and again.  order[] receives every chain front to back,     */
/* chain_start[] the offsets (n_chains + 1 entries).  Returns n_chains.        */
/* ------------------------------------------------------------------------- */
int64_t rdo_order(const float* S, int64_t ns, int dim, float r2, int32_t* order,
                  int32_t* chain_start)
{
    const float rsq = r2 * r2;
    unsigned char* alive = (unsigned char*)malloc((size_t)ns + 1);
    int32_t* deq = (int32_t*)malloc(sizeof(int32_t) * (size_t)(2 * ns + 1));
    memset(alive, 1, (size_t)ns + 1);
    int64_t out = 0, nch = 0;
    for (int64_t p = 0; p < ns; ++p) {
        if (!alive[p]) continue;
        alive[p] = 0;
        int64_t head = ns, tail = ns;
        deq[ns] = (int32_t)p;
        for (;;) {
            int64_t hit = -1;
            int front = 0;
            for (int64_t j = p + 1; j < ns; ++j) {
                if (!alive[j]) continue;
                if (sqdist(S + j * dim, S + (int64_t)deq[head] * dim, dim) <= rsq) {
                    hit = j; front = 1; break;
                }
                if (sqdist(S + j * dim, S + (int64_t)deq[tail] * dim, dim) <= rsq) {
                    hit = j; break;
                }
            }
            if (hit < 0) break;
            alive[hit] = 0;
            if (front) deq[--head] = (int32_t)hit;
            else deq[++tail] = (int32_t)hit;
        }
        chain_start[nch++] = (int32_t)out;
        for (int64_t k = head; k <= tail; ++k) order[out++] = deq[k];
    }
    chain_start[nch] = (int32_t)out;
    free(alive);
    free(deq);
    return nch;
}

/* ------------------------------------------------------------------------- */
/* rd/utils/assessment_quality.hpp in float, as the reference computes it.    */
/* ------------------------------------------------------------------------- */

/* :156-205 distance(): sqrt of the smallest squared distance from p to set B
 * (strict < over B in order; FLT_MAX when B is empty). */
static float q_distance(const float* p, const float* B, int64_t nb, int dim)
{
    float nearest = 3.402823466e+38f;
    for (int64_t k = 0; k < nb; ++k) {
        const float d = sqdist(p, B + k * dim, dim);
        if (d < nearest) nearest = d;
    }
    return sqrtf(nearest);
}

/* :207-222 setDistance(): the largest of those over A */
static float q_set_distance(const float* A, int64_t na, const float* B, int64_t nb, int dim)
{
    float mx = -3.402823466e+38f;
    for (int64_t i = 0; i < na; ++i) {
        const float d = q_distance(A + i * dim, B, nb, dim);
        if (d > mx) mx = d;
    }
    return mx;
}

/* :91-121 hausdorffDistance(): -1 for an empty test set */
float rdo_hausdorff_f32(const float* T, int64_t nt, const float* I, int64_t ni, int dim)
{
    if (nt <= 0) return -1.0f;
    const float ab = q_set_distance(T, nt, I, ni, dim);
    const float ba = q_set_distance(I, ni, T, nt, dim);
    return ab > ba ? ab : ba;
}

static int cmp_float(const void* a, const void* b)
{
    const float x = *(const float*)a, y = *(const float*)b;
    return (x > y) - (x < y);
}

/* :123-154 setDistanceStats(): distances of every source point to the ideal
 * set, sorted; min, max, median = sorted[n/2], average = float sum in sorted
 * order / n.  out = {median, avg, min, max}. */
void rdo_distance_stats_f32(const float* S, int64_t n, const float* I, int64_t ni, int dim,
                            float* out)
{
    float* d = (float*)malloc(sizeof(float) * (size_t)(n + 1));
    for (int64_t i = 0; i < n; ++i) d[i] = q_distance(S + i * dim, I, ni, dim);
    qsort(d, (size_t)n, sizeof(float), cmp_float);
    float avg = 0.0f;
    for (int64_t i = 0; i < n; ++i) avg += d[i];
    out[0] = d[n / 2];
    out[1] = avg / (float)n;
    out[2] = d[0];
    out[3] = d[n - 1];
    free(d);
}

/* :295-375 RDSegmentAssessmentQuality: the distance of every test point to the
 * x axis, sqrt(sum over d >= 1 of x_d^2) (0 when that sum is 0), and its
 * largest value; -1 for an empty test set. */
float rdo_segment_hausdorff_f32(const float* T, int64_t nt, int dim)
{
    if (nt <= 0) return -1.0f;
    float mx = -3.402823466e+38f;
    for (int64_t i = 0; i < nt; ++i) {
        float s = 0.0f;
        for (int k = 1; k < dim; ++k) s += T[i * dim + k] * T[i * dim + k];
        const float d = (s > 0.0f) ? sqrtf(s) : 0.0f;
        if (d > mx) mx = d;
    }
    return mx;
}
