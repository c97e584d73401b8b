// rd_tiled.hpp -- extended-tile tiled ridge detection on top of the batch engine.
//
// Semantics are those of the reference CPU implementation
// rd::tiled::tiledRidgeDetection<EXT_TILE_TREE_MIXED_RD> (rd/cpu/tiled/rd_tiled.hpp:1217-1374)
// over rd::tiled::TiledGroupTree<EXTENDED_TILE> (rd/cpu/tiled/grouped_tile_tree.inl):
//   * global bounding box; a uniform grid of tiles_per_dim tiles, dimension 0
//     fastest; tile c spans [min + c*step, min + (c+1)*step) per dimension, the
//     last one ending at the global max (grouped_tile_tree.inl:147-213);
//   * a point is an own point of the tile that holds it (min <= x < max) and a
//     halo point of every other tile whose box grown by r1 holds it
//     (rd/utils/bounding_box.hpp:335-375); both lists keep input order;
//   * tiles with 0 or 1 own points are dropped (:216-244); a tile with at least
//     max_tile_capacity own points is half-split along dimension level % dim,
//     recursively, over its own points then its halo (:247-330);
//   * every leaf chooses among its own points and evolves its chosen points over
//     its own points followed by its halo; all leaves are decimated together in
//     leaf order with decimateNoCopy semantics; repeat until the total count is
//     stable; the result is the leaves' chosen points in pre-order.
//
// Device side: bounding box, per-point tile/halo emission, a stable key sort
// that groups every tile's own points and halo points in input order, and the
// gather of the packed per-leaf point arrays the engine evolves.  Oversize tiles
// (own points >= max_tile_capacity) are split on the host with the same rules.
#pragma once

#include "rd_engine_host.hpp"

#include <cstdint>
#include <memory>
#include <vector>

namespace rdb {

struct TiledTimers {
    float whole_ms = 0, build_ms = 0, rd_ms = 0, refine_ms = 0;
};

class TiledRunner {
public:
    // d_points: n packed ROW_MAJOR points on the device (kept by the caller)
    int run(const float* d_points, int64_t n, int dim, float r1, float r2, int64_t cap,
            const int32_t* tiles_per_dim, bool use_graph, cudaStream_t st);

    int64_t ns() const { return ns_; }
    int64_t n_leaves() const { return (int64_t)leaf_ns_.size(); }
    const float* result() const { return bOut_.as<float>(); }  // ns x dim, leaf pre-order
    float* result_mut() { return bOut_.as<float>(); }
    // after an in-place change of the result (end-phase refinement)
    void set_result_count(int64_t ns) { ns_ = ns; }
    void add_refinement_time(float ms) { tm_.refine_ms = ms; tm_.whole_ms += ms; }
    const TiledTimers& timers() const { return tm_; }
    const RunStats& stats() const { return eng_.stats(); }
    // host-loop runs time every fused tile-evolve launch (RunStats.assign_ms)
    void set_profiling(bool on) { eng_.profile_assign = on; }
    std::string last_error;
    // false: RD_MIXED (local evolve, global decimation); true: RD_LOCAL (a full
    // ridge detection inside every leaf)
    bool local_policy = false;

private:
    int fail(const char* what, cudaError_t e);
    Engine eng_;
    DevBuf bBox_, bBounds_, bCnt_, bOff_, bKeys_, bVals_, bKeys2_, bVals2_, bTemp_, bSeg_;
    DevBuf bExtra_, bOut_, bTab_;
    // subdivision of oversize tiles on the device: per-level scratch, and the
    // sorted point lists of every level (the leaves' lists stay there)
    DevBuf bSplitTab_, bSplitBox_, bSplitE_, bSplitCode_, bSplitCnt_, bSplitOff_, bSplitK_,
        bSplitV_, bSplitK2_, bSplitSeg_;
    std::vector<std::unique_ptr<DevBuf>> split_bufs_;
    std::vector<int32_t> leaf_ns_;
    int64_t ns_ = 0;
    TiledTimers tm_;
};

}  // namespace rdb
