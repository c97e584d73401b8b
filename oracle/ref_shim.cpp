/*
 * ref_shim.cpp -- TEST INFRASTRUCTURE ONLY (oracle side, never the product).
 *
 * A thin extern "C" wrapper that is compiled TOGETHER WITH the reference's own
 * CPU headers (include path points into the reference checkout; nothing from
 * there is copied into this repository).  The resulting shared objects live in
 * oracle/_ref/ (git-ignored) and are used only to
 *   (1) pin the plain-C restatement in oracle/rd_oracle.c against the
 *       reference's real code on seeded inputs (tests/golden/make_golden.py),
 *   (2) time the reference's OpenMP CPU path as the CPU baseline in bench.py.
 *
 * Two builds come out of this one file (see oracle/Makefile):
 *   librdref.so      serial   (no RD_USE_OPENMP)  -> deterministic, bit-exact oracle
 *   librdref_omp.so  OpenMP   (-DRD_USE_OPENMP)   -> timed CPU baseline
 *
 * Entry points mirror, one to one, the reference functions they call:
 *   rd::choose                     rd/cpu/brute_force/choose.hpp:37
 *   rd::detail::calculateClosestSphereCenter / shiftTowardMassCenter
 *                                  rd/cpu/brute_force/evolve.hpp:33,130
 *   rd::evolve / rd::evolve_omp    rd/cpu/brute_force/evolve.hpp:293,238
 *   rd::decimate                   rd/cpu/brute_force/decimate.hpp:41
 *   rd::decimateNoCopy             rd/cpu/brute_force/decimate.hpp:85
 *   rd::RidgeDetection<float>      rd/cpu/brute_force/ridge_detection.inl:68
 *   rd::tiled::tiledRidgeDetection<EXT_TILE_TREE_MIXED_RD>
 *                                  rd/cpu/tiled/rd_tiled.hpp:1766
 */
#include "rd/cpu/brute_force/ridge_detection.hpp"
#include "rd/cpu/brute_force/choose.hpp"
#include "rd/cpu/brute_force/evolve.hpp"
#include "rd/cpu/brute_force/decimate.hpp"
#include "rd/cpu/tiled/rd_tiled.hpp"
#include "rd/cpu/brute_force/order.hpp"
#include "rd/utils/samples_set.hpp"
#include "rd/utils/assessment_quality.hpp"

#include <cstdint>
#include <cstring>
#include <list>
#include <vector>

#if defined(RD_USE_OPENMP)
#include <omp.h>
#endif

extern "C" {

int ref_is_openmp(void)
{
#if defined(RD_USE_OPENMP)
    return 1;
#else
    return 0;
#endif
}

int ref_max_threads(void)
{
#if defined(RD_USE_OPENMP)
    return omp_get_num_procs();
#else
    return 1;
#endif
}

/* rd::choose -- returns ns; S must hold np*dim floats. */
int64_t ref_choose(const float* P, int64_t np, int dim, float r1, float* S)
{
    std::list<float*> lst;
    size_t ns = 0;
    rd::choose<float>(P, S, lst, (size_t)np, ns, (size_t)dim, r1);
    return (int64_t)ns;
}

/* One evolve pass: closest-sphere sums + shift.  sums/cnt are outputs
 * (zeroed here first, as evolve.hpp:316-317 does).  Returns contFlag. */
int ref_evolve_pass(const float* P, int64_t np, float* S, int64_t ns, int dim,
                    float r1, float* sums, int32_t* cnt)
{
    float rSqr = r1 * r1;
    std::memset(sums, 0, sizeof(float) * (size_t)ns * (size_t)dim);
    std::memset(cnt, 0, sizeof(int32_t) * (size_t)ns);
    rd::detail::calculateClosestSphereCenter<float>(P, S, sums, cnt, (size_t)np,
                                                    (size_t)ns, (size_t)dim, rSqr);
    int contFlag = 0;
    rd::detail::shiftTowardMassCenter<float>(S, sums, cnt, (size_t)ns, (size_t)dim,
                                             contFlag);
    return contFlag;
}

/* `passes` evolve passes exactly as the loop body of rd::evolve_omp
 * (evolve.hpp:258-286) runs them: an OpenMP region that zeroes the sums and
 * calls calculateClosestSphereCenter_omp, then shiftTowardMassCenter_omp.
 * Used to time a bounded sample of the reference's OpenMP evolve.  Returns
 * the continue flag of the last pass. */
int ref_evolve_passes_omp(const float* P, int64_t np, float* S, int64_t ns, int dim, float r1,
                          int threads, int passes)
{
    float rSqr = r1 * r1;
    std::vector<float> cordSums((size_t)(ns * dim) + 1);
    std::vector<int> cnt((size_t)ns + 1);
    int contFlag = 0;
#if defined(RD_USE_OPENMP)
    const int nt = threads > 0 ? threads : omp_get_num_procs();
    for (int p = 0; p < passes; ++p) {
        float* cs = cordSums.data();
        int* sc = cnt.data();
        #pragma omp parallel num_threads(nt)
        {
            rd::fillTable_omp(cs, 0.f, (size_t)(ns * dim));
            rd::fillTable_omp(sc, 0, (size_t)ns);
            rd::detail::calculateClosestSphereCenter_omp<float>(P, S, cs, sc, (size_t)np,
                                                                (size_t)ns, (size_t)dim, rSqr);
        }
        contFlag = 0;
        rd::detail::shiftTowardMassCenter_omp<float>(S, cs, sc, (size_t)ns, (size_t)dim,
                                                     contFlag, nt);
    }
#else
    (void)threads;
    for (int p = 0; p < passes; ++p) {
        std::fill(cordSums.begin(), cordSums.end(), 0.f);
        std::fill(cnt.begin(), cnt.end(), 0);
        rd::detail::calculateClosestSphereCenter<float>(P, S, cordSums.data(), cnt.data(),
                                                        (size_t)np, (size_t)ns, (size_t)dim, rSqr);
        contFlag = 0;
        rd::detail::shiftTowardMassCenter<float>(S, cordSums.data(), cnt.data(), (size_t)ns,
                                                 (size_t)dim, contFlag);
    }
#endif
    return contFlag;
}

/* rd::evolve (serial) or rd::evolve_omp (threads > 0, OpenMP build only). */
void ref_evolve(const float* P, int64_t np, float* S, int64_t ns, int dim, float r1,
                int threads)
{
#if defined(RD_USE_OPENMP)
    if (threads > 0) {
        rd::evolve_omp<float>(P, S, (size_t)np, (size_t)ns, (size_t)dim, r1, threads);
        return;
    }
#endif
    (void)threads;
    rd::evolve<float>(P, S, (size_t)np, (size_t)ns, (size_t)dim, r1);
}

/* rd::decimate over S[0..ns) in array order; compacts S; returns new ns. */
int64_t ref_decimate(float* S, int64_t ns, int dim, float r2)
{
    std::list<float*> lst;
    for (int64_t k = 0; k < ns; ++k) lst.push_back(S + k * dim);
    size_t cnt = (size_t)ns;
    rd::decimate<float>(S, lst, cnt, (size_t)dim, r2);
    return (int64_t)cnt;
}

/* rd::decimateNoCopy over nseg consecutive segments of S (segment k holds
 * seg_cnt[k] points).  Survivors are compacted per segment in place at the
 * front of the whole S (segments stay in order); seg_cnt is updated.
 * Returns the new total count. */
int64_t ref_decimate_nocopy(float* S, int64_t nseg, int64_t* seg_cnt, int dim, float r2)
{
    std::vector<std::list<float*>> lists((size_t)nseg);
    std::list<std::list<float*>*> g;
    size_t total = 0;
    float* p = S;
    for (int64_t s = 0; s < nseg; ++s) {
        for (int64_t k = 0; k < seg_cnt[s]; ++k) { lists[s].push_back(p); p += dim; }
        total += (size_t)seg_cnt[s];
        g.push_back(&lists[s]);
    }
    rd::decimateNoCopy<float>(g, total, (size_t)dim, r2);
    std::vector<float> out;
    out.reserve(total * (size_t)dim);
    for (int64_t s = 0; s < nseg; ++s) {
        seg_cnt[s] = (int64_t)lists[s].size();
        for (float* q : lists[s]) out.insert(out.end(), q, q + dim);
    }
    std::memcpy(S, out.data(), out.size() * sizeof(float));
    return (int64_t)total;
}

/* rd::RidgeDetection<float>::ridgeDetection.  threads == 0 -> noOMP()
 * (serial, deterministic); threads > 0 -> ompSetNumThreads(threads) (only
 * meaningful in the OpenMP build).  S must hold np*dim floats. */
int64_t ref_bf_ridge(const float* P, int64_t np, int dim, float r1, float r2, float* S,
                     int threads)
{
    rd::RidgeDetection<float> rd;
    if (threads <= 0) rd.noOMP();
    else rd.ompSetNumThreads(threads);
    rd.ridgeDetection(P, (size_t)np, S, r1, r2, (size_t)dim);
    return (int64_t)rd.ns_;
}

/* rd::tiled::tiledRidgeDetection<EXT_TILE_TREE_MIXED_RD> without end-phase
 * refinement.  S_out must hold np*dim floats.  Returns ns; times[4] gets
 * (whole, tree, rdTiles, refinement) in ms. */
int64_t ref_tiled_ridge(const float* P, int64_t np, int dim, float r1, float r2,
                        int64_t max_tile_capacity, const int64_t* tiles_per_dim,
                        int threads, int refinement, float* S_out, float* times)
{
    rd::tiled::rdTiledData<float> dp;
    dp.dim = (size_t)dim;
    dp.np = (size_t)np;
    dp.r1 = r1;
    dp.r2 = r2;
    dp.P = P;
    dp.maxTileCapacity = (size_t)max_tile_capacity;
    dp.nTilesPerDim.assign(tiles_per_dim, tiles_per_dim + dim);
    auto t = rd::tiled::tiledRidgeDetection<rd::tiled::EXT_TILE_TREE_MIXED_RD>(
        dp, threads > 0 ? threads : 1, refinement != 0, false, false);
    if (times) {
        times[0] = std::get<0>(t);
        times[1] = std::get<1>(t);
        times[2] = std::get<2>(t);
        times[3] = std::get<3>(t);
    }
    std::memcpy(S_out, dp.S.data(), dp.S.size() * sizeof(float));
    return (int64_t)dp.ns;
}

// rd::Samples<float>::loadFromFile (rd/utils/samples_set.hpp:254-294): the
// reference's text cloud reader.  The file is found as <directory of the
// running executable>/<folder><filename>, as the reference resolves it
// (rd/utils/utilities.hpp:149-184).  Returns the point count, -1 on a thrown
// error, -2 when cap is too small; *dim receives the dimension.
int64_t ref_load_text(const char* folder, const char* filename, float* out, int64_t cap,
                      int* dim)
{
    try {
        rd::Samples<float> s;
        s.loadFromFile(filename, folder);
        *dim = (int)s.dim_;
        if ((int64_t)(s.size_ * s.dim_) > cap) return -2;
        std::memcpy(out, s.samples_, sizeof(float) * s.size_ * s.dim_);
        return (int64_t)s.size_;
    } catch (...) {
        return -1;
    }
}

// rd::RDAssessmentQuality<float> (rd/utils/assessment_quality.hpp) on a given
// ideal pattern: the reference generates its patterns from unseeded random
// draws, so the shim sets the protected pattern directly.
struct ShimQuality : rd::RDAssessmentQuality<float> {
    ShimQuality(const float* ideal, size_t n, size_t dim) : rd::RDAssessmentQuality<float>(n, dim)
    {
        idealPattern.assign(ideal, ideal + n * dim);
    }
};

float ref_hausdorff_f32(const float* T, int64_t nt, const float* I, int64_t ni, int dim)
{
    ShimQuality q(I, (size_t)ni, (size_t)dim);
    return q.hausdorffDistance(std::vector<float>(T, T + nt * dim));
}

void ref_distance_stats_f32(const float* S, int64_t n, const float* I, int64_t ni, int dim,
                            float* out)
{
    ShimQuality q(I, (size_t)ni, (size_t)dim);
    q.setDistanceStats(std::vector<float>(S, S + n * dim), out[0], out[1], out[2], out[3]);
}

float ref_segment_hausdorff_f32(const float* T, int64_t nt, int dim)
{
    rd::RDSegmentAssessmentQuality<float> q(0, (size_t)dim);
    return q.hausdorffDistance(std::vector<float>(T, T + nt * dim));
}

// rd::orderSamples (rd/cpu/brute_force/order.hpp:45) with the condition the
// brute-force class passes (ridge_detection.inl:148-168); chains flattened to
// point indices, front to back, with their start offsets.
int64_t ref_order(const float* S, int64_t ns, int dim, float r2, int32_t* order,
                  int32_t* chain_start)
{
    const float r2Sqr = r2 * r2;
    auto chains = rd::orderSamples<float>(S, (size_t)dim, (size_t)ns,
        [&r2Sqr](float const* p1, float const* p2, size_t d) -> bool {
            return rd::squareEuclideanDistance(p1, p2, d) <= r2Sqr;
        });
    int64_t out = 0, nch = 0;
    for (const auto& ch : chains) {
        chain_start[nch++] = (int32_t)out;
        for (const float* q : ch) order[out++] = (int32_t)((q - S) / dim);
    }
    chain_start[nch] = (int32_t)out;
    return nch;
}

}  // extern "C"
