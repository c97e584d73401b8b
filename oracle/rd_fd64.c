/*
 * rd_fd64.c -- FP64 evaluation of the evolve adjoint's forward map and central
 * finite differences of its loss, with every assignment recomputed.
 *
 * TEST INFRASTRUCTURE ONLY (part of librdoracle.so, the checker); the product
 * never links it.
 *
 * The map is the adjoint's forward (no reference counterpart; its assignment
 * rule is rd/cpu/brute_force/evolve.hpp:43-76 evaluated in double): at pass t
 * every cloud point goes to its nearest chosen point, the lowest index winning
 * a tie, when that squared distance is <= r1*r1; each chosen point with
 * members becomes the mean of its members (double sum in index order divided
 * by the count), one without members keeps its position.  The loss is
 * L = sum_k <W_k, S^iters_k>.
 *
 * Nearest-point searches go through a hashed grid of cell edge r1: the nearest
 * chosen point within r1 of a point lies in the 3^dim cells around it, so only
 * those cells are visited (every candidate is tested with the exact distance,
 * the grid only prunes).
 *
 * Finite differences.  Moving one coordinate of cloud point i by +-h changes,
 * at pass t, only the chosen points whose member sums contain point i and the
 * empty clusters that carry such a change forward.  So the perturbed run is
 * evaluated exactly by recomputing, at every pass, the assignment of point i
 * and of every point within r1 of a changed chosen point (old or new
 * position) -- no other point can change its nearest chosen point or its
 * membership -- and the means of the clusters that point i belongs to.  If any
 * recomputed assignment differs from the unperturbed run, the coordinate is
 * reported as lying on a ball or Voronoi boundary (the difference quotient
 * would then not be a derivative) and no value is returned.
 */
#include "rd_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#define CELL_BIAS (1 << 20)
#define CELL_MAX ((1 << 21) - 1)

static inline int64_t cell_of(double x, double inv)
{
    double c = floor(x * inv);
    if (!(c > -CELL_BIAS)) c = -CELL_BIAS;    /* also maps NaN to the lowest cell */
    if (c > CELL_MAX - CELL_BIAS) c = CELL_MAX - CELL_BIAS;
    return (int64_t)c + CELL_BIAS;
}

static inline uint64_t cell_hash(const int64_t* c, int dim)
{
    uint64_t h = 0x9E3779B97F4A7C15ull;
    for (int d = 0; d < dim; ++d) {
        h ^= (uint64_t)c[d] + 0x632BE59BD9B4E019ull + (h << 6) + (h >> 2);
        h *= 0xFF51AFD7ED558CCDull;
    }
    return h ^ (h >> 29);
}

typedef struct grid64 {
    int dim;
    double inv;
    int64_t tsize;     /* power of two */
    int32_t* head;     /* tsize chains */
    int32_t* next;     /* one link per item */
} grid64;

static int grid_build(grid64* g, const double* X, int64_t n, int dim, double cell)
{
    g->dim = dim;
    g->inv = 1.0 / cell;
    g->tsize = 64;
    while (g->tsize < 2 * n) g->tsize <<= 1;
    g->head = (int32_t*)malloc(sizeof(int32_t) * (size_t)g->tsize);
    g->next = (int32_t*)malloc(sizeof(int32_t) * (size_t)(n + 1));
    if (!g->head || !g->next) return 1;
    for (int64_t b = 0; b < g->tsize; ++b) g->head[b] = -1;
    /* insert in reverse so every chain lists its items in increasing index */
    for (int64_t k = n - 1; k >= 0; --k) {
        int64_t c[4];
        for (int d = 0; d < dim; ++d) c[d] = cell_of(X[k * dim + d], g->inv);
        const int64_t b = (int64_t)(cell_hash(c, dim) & (uint64_t)(g->tsize - 1));
        g->next[k] = g->head[b];
        g->head[b] = (int32_t)k;
    }
    return 0;
}

static void grid_free(grid64* g)
{
    free(g->head);
    free(g->next);
}

static inline double sqdist64(const double* a, const double* b, int dim)
{
    double acc = 0.0;
    for (int d = 0; d < dim; ++d) {
        const double t = a[d] - b[d];
        acc += t * t;
    }
    return acc;
}

/* Visits the 3^dim cells around p and calls fn(item) for every item of their
 * chains (an item can be visited more than once when chains collide). */
#define GRID_VISIT(g, p, ITEM, BODY)                                                 \
    do {                                                                             \
        int64_t c0_[4], c_[4];                                                       \
        for (int d_ = 0; d_ < (g)->dim; ++d_) c0_[d_] = cell_of((p)[d_], (g)->inv);  \
        int nb_ = 1;                                                                 \
        for (int d_ = 0; d_ < (g)->dim; ++d_) nb_ *= 3;                              \
        for (int o_ = 0; o_ < nb_; ++o_) {                                           \
            int r_ = o_;                                                             \
            for (int d_ = 0; d_ < (g)->dim; ++d_) {                                  \
                c_[d_] = c0_[d_] + (r_ % 3) - 1;                                     \
                r_ /= 3;                                                             \
            }                                                                        \
            const int64_t b_ =                                                       \
                (int64_t)(cell_hash(c_, (g)->dim) & (uint64_t)((g)->tsize - 1));      \
            for (int32_t ITEM = (g)->head[b_]; ITEM >= 0; ITEM = (g)->next[ITEM]) { BODY } \
        }                                                                            \
    } while (0)

/* nearest chosen point of p within r1 (lowest index on ties), else -1 */
static int32_t nearest64(const grid64* g, const double* S, const double* p, double rsq)
{
    double best = INFINITY;
    int32_t bk = -1;
    GRID_VISIT(g, p, k, {
        const double dd = sqdist64(S + (int64_t)k * g->dim, p, g->dim);
        if (dd < best || (dd == best && k < bk)) { best = dd; bk = k; }
    });
    return (bk >= 0 && best <= rsq) ? bk : -1;
}

int rdo_forward64(const double* P, int64_t np, const double* S0, int64_t ns, int dim,
                  double r1, int iters, double* S_all, int32_t* keys, int32_t* cnt)
{
    const double rsq = r1 * r1;
    double* sums = (double*)malloc(sizeof(double) * (size_t)(ns * dim + 1));
    if (!sums) return 1;
    memcpy(S_all, S0, sizeof(double) * (size_t)(ns * dim));
    for (int t = 0; t < iters; ++t) {
        const double* S = S_all + (int64_t)t * ns * dim;
        double* Sn = S_all + (int64_t)(t + 1) * ns * dim;
        int32_t* kt = keys + (int64_t)t * np;
        int32_t* ct = cnt + (int64_t)t * ns;
        grid64 g;
        if (grid_build(&g, S, ns, dim, r1)) { free(sums); return 1; }
        for (int64_t i = 0; i < np; ++i) kt[i] = nearest64(&g, S, P + i * dim, rsq);
        grid_free(&g);
        memset(sums, 0, sizeof(double) * (size_t)(ns * dim));
        memset(ct, 0, sizeof(int32_t) * (size_t)ns);
        for (int64_t i = 0; i < np; ++i) {
            const int32_t k = kt[i];
            if (k < 0) continue;
            ct[k] += 1;
            for (int d = 0; d < dim; ++d) sums[(int64_t)k * dim + d] += P[i * dim + d];
        }
        for (int64_t k = 0; k < ns; ++k)
            for (int d = 0; d < dim; ++d)
                Sn[k * dim + d] = ct[k] ? sums[k * dim + d] / (double)ct[k] : S[k * dim + d];
    }
    free(sums);
    return 0;
}

/* a chosen point whose position differs from the unperturbed run */
typedef struct moved64 {
    int32_t k;
    double x[4];
} moved64;

/* one signed run; out_moved receives the final changed chosen points.
 * Returns 0, 1 when an assignment changed, 2 on allocation failure. */
static int perturbed_run(const double* P, int64_t np, const double* S_all, const int32_t* keys,
                         const int32_t* cnt, int64_t ns, int dim, double r1, int iters,
                         const grid64* pg, int64_t i, int d, int64_t s0_row, double step,
                         moved64* moved, int* n_moved)
{
    const double rsq = r1 * r1;
    double pi[4];
    for (int e = 0; e < dim; ++e) pi[e] = P[i * dim + e];
    pi[d] += step;
    int nm = 0;
    if (s0_row >= 0) {
        moved[0].k = (int32_t)s0_row;
        for (int e = 0; e < dim; ++e) moved[0].x[e] = S_all[s0_row * dim + e];
        moved[0].x[d] += step;
        nm = 1;
    }
    double* St = (double*)malloc(sizeof(double) * (size_t)(ns * dim + 1));
    if (!St) return 2;
    int rc = 0;
    for (int t = 0; t < iters && rc == 0; ++t) {
        const double* Sb = S_all + (int64_t)t * ns * dim;
        const int32_t* kt = keys + (int64_t)t * np;
        const int32_t* ct = cnt + (int64_t)t * ns;
        memcpy(St, Sb, sizeof(double) * (size_t)(ns * dim));
        for (int m = 0; m < nm; ++m)
            for (int e = 0; e < dim; ++e) St[(int64_t)moved[m].k * dim + e] = moved[m].x[e];
        grid64 sg;
        if (grid_build(&sg, St, ns, dim, r1)) { rc = 2; break; }
        if (nearest64(&sg, St, pi, rsq) != kt[i]) rc = 1;
        for (int m = 0; m < nm && rc == 0; ++m) {
            const int32_t k = moved[m].k;
            for (int side = 0; side < 2 && rc == 0; ++side) {
                const double* c = side ? moved[m].x : Sb + (int64_t)k * dim;
                GRID_VISIT(pg, c, j, {
                    if (rc == 0 && j != i && nearest64(&sg, St, P + (int64_t)j * dim, rsq) != kt[j])
                        rc = 1;
                });
            }
        }
        grid_free(&sg);
        if (rc) break;
        /* the next pass: point i's cluster gets a new mean; empty clusters
         * carry their changed position; every other cluster is unchanged */
        int nn = 0;
        moved64 next[8];
        const int32_t ki = kt[i];
        if (ki >= 0) {
            double s[4] = {0, 0, 0, 0};
            for (int64_t j = 0; j < np; ++j) {
                if (kt[j] != ki) continue;
                const double* pj = (j == i) ? pi : P + j * dim;
                for (int e = 0; e < dim; ++e) s[e] += pj[e];
            }
            next[nn].k = ki;
            for (int e = 0; e < dim; ++e) next[nn].x[e] = s[e] / (double)ct[ki];
            ++nn;
        }
        for (int m = 0; m < nm; ++m) {
            if (ct[moved[m].k] != 0 || moved[m].k == ki) continue;
            if (nn == 8) { rc = 1; break; }  /* more carried changes than tracked */
            next[nn++] = moved[m];
        }
        nm = nn;
        for (int m = 0; m < nm; ++m) moved[m] = next[m];
    }
    free(St);
    *n_moved = nm;
    return rc;
}

int rdo_fd64(const double* P, int64_t np, const double* S_all, const int32_t* keys,
             const int32_t* cnt, int64_t ns, int dim, double r1, int iters, const double* W,
             int64_t i, int d, int64_t s0_row, double h, double* fd)
{
    if (dim < 1 || dim > 4 || i < 0 || i >= np || d < 0 || d >= dim) return 2;
    grid64 pg;
    if (grid_build(&pg, P, np, dim, r1)) return 2;
    moved64 mp[8], mm[8];
    int np_ = 0, nm_ = 0;
    int rc = perturbed_run(P, np, S_all, keys, cnt, ns, dim, r1, iters, &pg, i, d, s0_row, h,
                           mp, &np_);
    if (rc == 0)
        rc = perturbed_run(P, np, S_all, keys, cnt, ns, dim, r1, iters, &pg, i, d, s0_row, -h,
                           mm, &nm_);
    grid_free(&pg);
    if (rc) return rc;
    /* (L(+h) - L(-h)) / 2h over the chosen points that differ in either run */
    const double* Sf = S_all + (int64_t)iters * ns * dim;
    double acc = 0.0;
    for (int pass = 0; pass < 2; ++pass) {
        const moved64* a = pass ? mm : mp;
        const int na = pass ? nm_ : np_;
        for (int m = 0; m < na; ++m) {
            const int32_t k = a[m].k;
            /* count each chosen point once: in the +h list, or in the -h list
             * when the +h run left it unchanged */
            if (pass) {
                int seen = 0;
                for (int q = 0; q < np_; ++q) seen |= (mp[q].k == k);
                if (seen) continue;
            }
            const double* xp = Sf + (int64_t)k * dim;
            const double* xm = Sf + (int64_t)k * dim;
            for (int q = 0; q < np_; ++q) if (mp[q].k == k) xp = mp[q].x;
            for (int q = 0; q < nm_; ++q) if (mm[q].k == k) xm = mm[q].x;
            for (int e = 0; e < dim; ++e) acc += W[(int64_t)k * dim + e] * (xp[e] - xm[e]);
        }
    }
    *fd = acc / (2.0 * h);
    return 0;
}
