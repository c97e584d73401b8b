/*
 * rd_oracle.h -- CPU restatement of the reference's ridge-detection path.
 *
 * TEST INFRASTRUCTURE ONLY.  Only tests/, __graft_entry__.smoke() and the CPU
 * baseline leg of bench.py may load this library, and only as the checker; the
 * product path (ridgedetection_b200 + librd_b200.so) never calls it.
 *
 * Parity pin: every function here is checked against the reference's own CPU
 * code compiled from its sources (oracle/ref_shim.cpp -> oracle/_ref/) on seeded
 * inputs; the outputs of those runs are committed as tests/golden/*.npz by
 * tests/golden/make_golden.py, and tests/test_oracle.py asserts bit equality.
 *
 * Arithmetic is plain IEEE FP32 with contraction disabled (-ffp-contract=off),
 * in exactly the operation order of the reference:
 *   squared distance   t = a - b; acc += t*t, d = 0..dim-1, acc = 0  (rd_inner.hpp:42-49)
 *   argmin             strict '<', lowest index wins ties            (evolve.hpp:54-65)
 *   membership         min <= r1*r1                                   (evolve.hpp:66)
 *   shift test         |mc - c| > 2.f*|mc|*cnt*FLT_EPSILON            (evolve.hpp:151-153)
 */
#ifndef RD_ORACLE_H
#define RD_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct rdo_stats {
    int64_t outer_iters;    /* evolve->decimate rounds                         */
    int64_t evolve_passes;  /* assignment+shift passes, summed over rounds     */
    double  pairs;          /* sum over passes of (cloud points x chosen)      */
    int64_t ns_choose;      /* chosen count right after choose                 */
} rdo_stats;

int64_t rdo_choose(const float* P, int64_t np, int dim, float r1, float* S);

void rdo_assign(const float* P, int64_t np, const float* S, int64_t ns, int dim,
                float r1, int32_t* key);
void rdo_accumulate(const float* P, int64_t np, const int32_t* key, int64_t ns, int dim,
                    float* sums, int32_t* cnt);
int rdo_shift(float* S, const float* sums, const int32_t* cnt, int64_t ns, int dim);
int rdo_evolve_pass(const float* P, int64_t np, float* S, int64_t ns, int dim, float r1,
                    float* sums, int32_t* cnt, int32_t* key);
int64_t rdo_evolve(const float* P, int64_t np, float* S, int64_t ns, int dim, float r1,
                   int64_t max_passes, double* pairs);

int64_t rdo_decimate(float* S, int64_t ns, int dim, float r2);
int64_t rdo_decimate_seg(float* S, int64_t nseg, int64_t* seg_cnt, int dim, float r2);

int64_t rdo_ridge_bf(const float* P, int64_t np, int dim, float r1, float r2, float* S,
                     rdo_stats* st);

int64_t rdo_ridge_tiled(const float* P, int64_t np, int dim, float r1, float r2,
                        int64_t max_tile_capacity, const int64_t* tiles_per_dim,
                        float* S, int64_t* n_leaves, rdo_stats* st);

double rdo_hausdorff(const float* A, int64_t na, const float* B, int64_t nb, int dim);
int64_t rdo_ridge_tiled_policy(const float* P, int64_t np, int dim, float r1, float r2,
                               int64_t max_tile_capacity, const int64_t* tiles_per_dim,
                               int local, float* S, int64_t* n_leaves, rdo_stats* st);
float rdo_hausdorff_f32(const float* T, int64_t nt, const float* I, int64_t ni, int dim);
void rdo_distance_stats_f32(const float* S, int64_t n, const float* I, int64_t ni, int dim,
                            float* out);
float rdo_segment_hausdorff_f32(const float* T, int64_t nt, int dim);
int64_t rdo_order(const float* S, int64_t ns, int dim, float r2, int32_t* order,
                  int32_t* chain_start);

/* FP64 reverse pass of `iters` evolve passes with a frozen assignment
 * recomputed from the forward iterates.  See rd_oracle.c for the exact
 * definition.  grad_P gets dL/dP for L = sum_k <W_k, S_k(final)>. */
int rdo_evolve_adjoint(const float* P, int64_t np, const float* S0, int64_t ns, int dim,
                       float r1, int iters, const double* W, double* grad_P,
                       double* grad_S0, float* S_final);

/* FP64 forward of the evolve adjoint's map with recomputed assignments, and
 * central differences of its loss (rd_fd64.c).  S_all: (iters+1) x ns x dim,
 * keys: iters x np, cnt: iters x ns.  rdo_fd64 returns 0 with *fd set, 1 when
 * the +-h runs change an assignment (a boundary coordinate), 2 on bad input. */
int rdo_forward64(const double* P, int64_t np, const double* S0, int64_t ns, int dim,
                  double r1, int iters, double* S_all, int32_t* keys, int32_t* cnt);
int rdo_fd64(const double* P, int64_t np, const double* S_all, const int32_t* keys,
             const int32_t* cnt, int64_t ns, int dim, double r1, int iters, const double* W,
             int64_t i, int d, int64_t s0_row, double h, double* fd);

#ifdef __cplusplus
}
#endif
#endif
