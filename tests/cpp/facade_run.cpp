// Runs the C++ facade (include/rd_b200.hpp) the way the reference's own tests
// drive its GPU classes, on a cloud read from a file; writes the chosen points
// (ROW_MAJOR) for the caller to compare with a golden ridge.
//
//   facade_run bf_row|bf_col <dim> <n> <r1> <r2> <in.bin> <out.bin>
//   facade_run tiled|tiled_col <dim> <n> <r1> <r2> <in.bin> <out.bin> <cap> <t0> <t1> [<t2>]
//
// in.bin: n x dim float32, ROW_MAJOR.  out.bin: int64 count, then count x dim
// float32, ROW_MAJOR.
#include "rd_b200.hpp"

#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

using namespace rd::b200;

static std::vector<float> read_points(const char* path, size_t count)
{
    std::vector<float> v(count);
    FILE* f = std::fopen(path, "rb");
    if (!f || std::fread(v.data(), sizeof(float), count, f) != count) {
        std::fprintf(stderr, "cannot read %s\n", path);
        std::exit(2);
    }
    std::fclose(f);
    return v;
}

static void write_points(const char* path, const std::vector<float>& pts, int64_t n)
{
    FILE* f = std::fopen(path, "wb");
    if (!f) std::exit(3);
    std::fwrite(&n, sizeof(n), 1, f);
    std::fwrite(pts.data(), sizeof(float), pts.size(), f);
    std::fclose(f);
}

// the reference's brute-force test flow: fill dP_, ridgeDetection(), ns_ / dS_
template <int DIM, DataMemoryLayout L>
static std::vector<float> run_bf(const std::vector<float>& P, size_t n, float r1, float r2,
                                 int64_t& ns)
{
    bruteForce::RidgeDetection<float, DIM, L, L> rd(n, r1, r2);
    if (L == COL_MAJOR) {
        std::vector<float> cols(DIM * n);
        for (size_t i = 0; i < n; ++i)
            for (int d = 0; d < DIM; ++d) cols[d * n + i] = P[i * DIM + d];
        check_cuda(cudaMemcpy2D(rd.dP_, rd.pPitch_, cols.data(), n * sizeof(float),
                                n * sizeof(float), DIM, cudaMemcpyHostToDevice));
    } else {
        check_cuda(cudaMemcpy(rd.dP_, P.data(), n * DIM * sizeof(float), cudaMemcpyHostToDevice));
    }
    rd.ridgeDetection();
    ns = (int64_t)rd.ns_;
    std::vector<float> out(DIM * (size_t)ns);
    if (L == COL_MAJOR) {
        std::vector<float> cols(DIM * (size_t)ns);
        if (ns > 0)
            check_cuda(cudaMemcpy2D(cols.data(), ns * sizeof(float), rd.dS_, rd.sPitch_,
                                    ns * sizeof(float), DIM, cudaMemcpyDeviceToHost));
        for (int64_t i = 0; i < ns; ++i)
            for (int d = 0; d < DIM; ++d) out[i * DIM + d] = cols[d * ns + i];
    } else if (ns > 0) {
        check_cuda(cudaMemcpy(out.data(), rd.dS_, out.size() * sizeof(float), cudaMemcpyDeviceToHost));
    }
    return out;
}

// the reference's tiled flow: construct from host points, operator(), then
// getChosenPointsNum() / getChosenPoints()
template <int DIM, DataMemoryLayout L>
static std::vector<float> run_tiled(const std::vector<float>& P, int n, float r1, float r2, int cap,
                                    const int* tiles, int64_t& ns)
{
    tiled::RidgeDetection<DIM, ROW_MAJOR, L> rd(n, P.data());
    int tpd[DIM];
    for (int d = 0; d < DIM; ++d) tpd[d] = tiles[d];
    rd(r1, r2, cap, tpd, false);
    ns = rd.getChosenPointsNum();
    std::vector<float> got(DIM * (size_t)ns);
    if (ns > 0) rd.getChosenPoints(got.data());
    if (L != COL_MAJOR) return got;
    std::vector<float> out(got.size());
    for (int64_t i = 0; i < ns; ++i)
        for (int d = 0; d < DIM; ++d) out[i * DIM + d] = got[d * ns + i];
    return out;
}

template <int DIM>
static int run(const std::string& mode, int argc, char** argv)
{
    const size_t n = (size_t)std::atoll(argv[3]);
    const float r1 = (float)std::atof(argv[4]);
    const float r2 = (float)std::atof(argv[5]);
    const std::vector<float> P = read_points(argv[6], n * DIM);
    int64_t ns = 0;
    std::vector<float> out;
    if (mode == "bf_row") {
        out = run_bf<DIM, ROW_MAJOR>(P, n, r1, r2, ns);
    } else if (mode == "bf_col") {
        out = run_bf<DIM, COL_MAJOR>(P, n, r1, r2, ns);
    } else if (mode == "tiled" || mode == "tiled_col") {
        if (argc < 9 + DIM) return 4;
        const int cap = std::atoi(argv[8]);
        int tiles[DIM];
        for (int d = 0; d < DIM; ++d) tiles[d] = std::atoi(argv[9 + d]);
        out = (mode == "tiled") ? run_tiled<DIM, ROW_MAJOR>(P, (int)n, r1, r2, cap, tiles, ns)
                                : run_tiled<DIM, COL_MAJOR>(P, (int)n, r1, r2, cap, tiles, ns);
    } else {
        return 4;
    }
    write_points(argv[7], out, ns);
    return 0;
}

int main(int argc, char** argv)
{
    if (argc < 8) {
        std::fprintf(stderr, "usage: facade_run mode dim n r1 r2 in.bin out.bin [cap tiles...]\n");
        return 4;
    }
    const std::string mode = argv[1];
    const int dim = std::atoi(argv[2]);
    try {
        if (dim == 2) return run<2>(mode, argc, argv);
        if (dim == 3) return run<3>(mode, argc, argv);
    } catch (const std::exception& e) {
        std::fprintf(stderr, "%s\n", e.what());
        return 5;
    }
    return 4;
}
