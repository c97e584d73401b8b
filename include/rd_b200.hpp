// rd_b200.hpp -- header-only C++ facade of librd_b200.so with the class and
// member names of the reference's GPU classes, so that code written against
//   rd::gpu::bruteForce::RidgeDetection<T, DIM, IN, OUT>
//       (ridge_detection/rd/gpu/device/brute_force/simulation.cuh:35-112)
//   rd::gpu::tiled::RidgeDetection<DIM, IN, OUT, ALG, POLICY, TILE, T>
//       (ridge_detection/rd/gpu/device/tiled/simulation.cuh:41-241)
// switches by changing the namespace prefix to rd::b200 and linking
// librd_b200.so.  Only T = float is provided (the path computes in FP32).
//
// Brute force, as the reference is used (tests/test_rd_gpu_simulation/
// brute_force/simulation.cu:184-247): construct with (np, r1, r2), copy the
// cloud into the public device buffer dP_ (pitched for COL_MAJOR, pPitch_
// bytes per row), call ridgeDetection(), then getChosenSamplesCount(); the
// ns_ chosen points are in dS_ (pitched for COL_MAJOR, sPitch_ bytes).
#pragma once

#include "rd_c_api.h"

#include <cuda_runtime.h>

#include <cstddef>
#include <stdexcept>
#include <string>
#include <vector>

namespace rd {
namespace b200 {

// rd/utils/memory.h:21-26
enum DataMemoryLayout { ROW_MAJOR, COL_MAJOR, SOA };

inline void check(rd_status s)
{
    if (s != RD_OK) throw std::runtime_error(std::string("librd_b200: ") + rd_last_error());
}
inline void check_cuda(cudaError_t e)
{
    if (e != cudaSuccess) throw std::runtime_error(std::string("CUDA: ") + cudaGetErrorString(e));
}

namespace bruteForce {

template <typename T, int DIM, DataMemoryLayout IN_MEM_LAYOUT, DataMemoryLayout OUT_MEM_LAYOUT>
class RidgeDetection;

template <int DIM, DataMemoryLayout IN_MEM_LAYOUT, DataMemoryLayout OUT_MEM_LAYOUT>
class RidgeDetection<float, DIM, IN_MEM_LAYOUT, OUT_MEM_LAYOUT> {
    static_assert(IN_MEM_LAYOUT != SOA && OUT_MEM_LAYOUT != SOA, "ROW_MAJOR or COL_MAJOR");

public:
    size_t np_;
    size_t ns_;
    float r1_, r2_;
    float* dP_;        // device samples (caller fills), pitched if COL_MAJOR
    size_t pPitch_;    // bytes per row for COL_MAJOR input, 0 otherwise
    float* dS_;        // device chosen points after ridgeDetection()
    size_t sPitch_;    // bytes per row for COL_MAJOR output, 0 otherwise
    bool verbose_;

    RidgeDetection(size_t np, float r1, float r2, bool verbose = false)
        : np_(np), ns_(0), r1_(r1), r2_(r2), dP_(nullptr), pPitch_(0), dS_(nullptr),
          sPitch_(0), verbose_(verbose), h_(nullptr)
    {
        check(rd_bf_create(&h_, DIM, IN_MEM_LAYOUT == COL_MAJOR ? RD_COL_MAJOR : RD_ROW_MAJOR,
                           OUT_MEM_LAYOUT == COL_MAJOR ? RD_COL_MAJOR : RD_ROW_MAJOR,
                           (int64_t)np, r1, r2));
        if (IN_MEM_LAYOUT == COL_MAJOR)
            check_cuda(cudaMallocPitch((void**)&dP_, &pPitch_, np_ * sizeof(float) + 4, DIM));
        else
            check_cuda(cudaMalloc((void**)&dP_, np_ * DIM * sizeof(float) + 16));
        if (OUT_MEM_LAYOUT == COL_MAJOR)
            check_cuda(cudaMallocPitch((void**)&dS_, &sPitch_, np_ * sizeof(float) + 4, DIM));
        else
            check_cuda(cudaMalloc((void**)&dS_, np_ * DIM * sizeof(float) + 16));
    }
    virtual ~RidgeDetection()
    {
        if (h_) rd_bf_destroy(h_);
        if (dP_) cudaFree(dP_);
        if (dS_) cudaFree(dS_);
    }
    RidgeDetection(const RidgeDetection&) = delete;
    RidgeDetection& operator=(const RidgeDetection&) = delete;

    // choose -> (evolve -> decimate)* on dP_, result in dS_
    void ridgeDetection()
    {
        const int64_t pitch = (IN_MEM_LAYOUT == COL_MAJOR) ? (int64_t)(pPitch_ / sizeof(float)) : DIM;
        check(rd_bf_set_points(h_, dP_, pitch, 1, nullptr));
        check(rd_bf_run(h_, nullptr));
        getChosenSamplesCount();
        const int64_t spitch = (OUT_MEM_LAYOUT == COL_MAJOR) ? (int64_t)(sPitch_ / sizeof(float)) : DIM;
        check(rd_bf_get_points(h_, dS_, spitch, 1, nullptr));
    }
    void getChosenSamplesCount()
    {
        int64_t n = 0;
        check(rd_bf_get_count(h_, &n));
        ns_ = (size_t)n;
    }

private:
    rd_bf* h_;
};

}  // namespace bruteForce

namespace tiled {

// rd/gpu/agent/agent_tiled_ridge_detection.cuh:96-102
struct TiledRidgeDetectionTimers {
    float wholeTime;
    float rdTilesTime;
    float refinementTime;
    float buildTreeTime;
};

enum RidgeDetectionAlgorithm { RD_BRUTE_FORCE };
enum TiledRidgeDetectionPolicy { RD_LOCAL, RD_MIXED };
enum TileType { RD_EXTENDED_TILE };

template <int DIM, DataMemoryLayout IN_MEM_LAYOUT, DataMemoryLayout OUT_MEM_LAYOUT,
          RidgeDetectionAlgorithm ALG = RD_BRUTE_FORCE, TiledRidgeDetectionPolicy POLICY = RD_MIXED,
          TileType TILE = RD_EXTENDED_TILE, typename T = float>
class RidgeDetection {
    static_assert(sizeof(T) == 4, "float only");

public:
    // inputPoints: host, ROW_MAJOR (as the reference's constructor takes them)
    RidgeDetection(int pointsNum, const T* inputPoints, bool enableTiming = false,
                   bool debugSynchronous = false)
        : pointsNum_(pointsNum), chosenPointsNum_(0), h_(nullptr)
    {
        (void)enableTiming;
        (void)debugSynchronous;
        check(rd_tiled_create(&h_, DIM, RD_ROW_MAJOR,
                              OUT_MEM_LAYOUT == COL_MAJOR ? RD_COL_MAJOR : RD_ROW_MAJOR, pointsNum));
        check(rd_tiled_set_points(h_, inputPoints, 0, 0, nullptr));
        check(rd_tiled_set_policy(h_, POLICY == RD_LOCAL ? RD_TILED_LOCAL : RD_TILED_MIXED));
    }
    ~RidgeDetection()
    {
        if (h_) rd_tiled_destroy(h_);
    }
    RidgeDetection(const RidgeDetection&) = delete;
    RidgeDetection& operator=(const RidgeDetection&) = delete;

    void operator()(T r1, T r2, int maxTileCapacity, int tilesPerDim[DIM], bool endPhaseRefinement)
    {
        ridgeDetection(r1, r2, maxTileCapacity, tilesPerDim, endPhaseRefinement);
    }
    void ridgeDetection(T r1, T r2, int maxTileCapacity, int tilesPerDim[DIM],
                        bool endPhaseRefinement)
    {
        int32_t tpd[DIM];
        for (int d = 0; d < DIM; ++d) tpd[d] = tilesPerDim[d];
        check(rd_tiled_run(h_, r1, r2, maxTileCapacity, tpd, endPhaseRefinement ? 1 : 0, nullptr));
    }
    int getChosenPointsNum()
    {
        int64_t n = 0;
        check(rd_tiled_get_count(h_, &n));
        chosenPointsNum_ = (int)n;
        return chosenPointsNum_;
    }
    // host output; ROW_MAJOR or (OUT_MEM_LAYOUT) COL_MAJOR with n = chosen count
    void getChosenPoints(T* chosenPoints)
    {
        check(rd_tiled_get_points(h_, chosenPoints, 0, 0, nullptr));
    }
    TiledRidgeDetectionTimers getTimers()
    {
        TiledRidgeDetectionTimers t{};
        check(rd_tiled_get_timers(h_, &t.wholeTime, &t.buildTreeTime, &t.rdTilesTime,
                                  &t.refinementTime));
        return t;
    }

private:
    int pointsNum_;
    int chosenPointsNum_;
    rd_tiled* h_;
};

}  // namespace tiled

// Exact culling of the brute-force assignment (process-wide, on by default):
// the same keys as the all-pairs comparison of rd/cpu/brute_force/evolve.hpp:43-66,
// skipping chosen points that provably lie beyond r1.  Read when a run starts.
inline void setAssignCull(bool enable) { check(rd_set_assign_cull(enable ? 1 : 0)); }
inline bool assignCull()
{
    int e = 0;
    check(rd_get_assign_cull(&e));
    return e != 0;
}

// rd::orderSamples (rd/cpu/brute_force/order.hpp:45) with the brute-force
// class's condition (squared distance <= r2*r2), on the device: chains of
// point indices of the ns x DIM ROW_MAJOR device points dS, each chain front
// to back.  The reference returns a list of deques of point pointers; the
// indices here are (pointer - S) / DIM of those.
inline std::vector<std::vector<int>> orderSamples(const float* dS, int dim, long long ns, float r2,
                                                  cudaStream_t stream = nullptr)
{
    std::vector<std::vector<int>> chains;
    int32_t* dOrder = nullptr;
    int32_t* dStart = nullptr;
    check_cuda(cudaMalloc(&dOrder, sizeof(int32_t) * (size_t)(ns + 1)));
    check_cuda(cudaMalloc(&dStart, sizeof(int32_t) * (size_t)(ns + 1)));
    int64_t nch = 0;
    const rd_status s = rd_order_chains(dim, dS, ns, r2, dOrder, dStart, &nch, stream);
    std::vector<int32_t> order((size_t)ns), start((size_t)nch + 1);
    if (s == RD_OK) {
        check_cuda(cudaMemcpy(order.data(), dOrder, sizeof(int32_t) * (size_t)ns,
                              cudaMemcpyDeviceToHost));
        check_cuda(cudaMemcpy(start.data(), dStart, sizeof(int32_t) * (size_t)(nch + 1),
                              cudaMemcpyDeviceToHost));
    }
    cudaFree(dOrder);
    cudaFree(dStart);
    check(s);
    for (int64_t c = 0; c < nch; ++c)
        chains.emplace_back(order.begin() + start[(size_t)c], order.begin() + start[(size_t)c + 1]);
    return chains;
}

}  // namespace b200
}  // namespace rd
