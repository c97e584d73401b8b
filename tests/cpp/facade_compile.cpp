// Compile/link check of include/rd_b200.hpp: every method of the facade is
// instantiated; main() does not call them (no GPU needed to build).
#include "rd_b200.hpp"

#include <vector>

using namespace rd::b200;

static void use_bf()
{
    bruteForce::RidgeDetection<float, 3, COL_MAJOR, COL_MAJOR> rd(1000, 0.15f, 0.3f);
    rd.ridgeDetection();
    rd.getChosenSamplesCount();
    (void)rd.ns_;
    (void)rd.dS_;
    bruteForce::RidgeDetection<float, 2, ROW_MAJOR, ROW_MAJOR> rd2(1000, 0.3f, 0.6f);
    rd2.ridgeDetection();
}

static void use_order()
{
    float* dS = nullptr;
    auto chains = orderSamples(dS, 3, 0, 0.3f);
    (void)chains.size();
    setAssignCull(assignCull());
}

static void use_tiled()
{
    std::vector<float> pts(2000, 0.f);
    tiled::RidgeDetection<2, ROW_MAJOR, ROW_MAJOR> rd(1000, pts.data());
    int tiles[2] = {4, 4};
    rd(0.2f, 0.4f, 1001, tiles, false);
    std::vector<float> out(2 * (size_t)rd.getChosenPointsNum());
    rd.getChosenPoints(out.data());
    (void)rd.getTimers();
    tiled::RidgeDetection<2, ROW_MAJOR, ROW_MAJOR, tiled::RD_BRUTE_FORCE, tiled::RD_LOCAL> rl(1000, pts.data());
    rl(0.2f, 0.4f, 1001, tiles, true);
}

int main(int argc, char**)
{
    if (argc > 99) {
        use_bf();
        use_tiled();
        use_order();
    }
    return 0;
}
