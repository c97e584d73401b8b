// rd_adjoint.hpp -- evolve adjoint on top of the batch engine (see rd_adjoint.cu).
#pragma once

#include "rd_engine_host.hpp"

namespace rdb {

class AdjointRunner {
public:
    // Every pointer is a device pointer.  d_W: ns x dim doubles (dL/dS_final);
    // d_S_final (optional): ns x dim floats; d_gP: np x dim doubles;
    // d_gS0 (optional): ns x dim doubles.  checkpoint_every = 0 keeps every
    // pass's assignment; k > 0 keeps S every k passes and recomputes.
    int run(int dim, const float* d_P, int64_t np, const float* d_S0, int64_t ns, float r1,
            int iters, int checkpoint_every, const double* d_W, float* d_S_final, double* d_gP,
            double* d_gS0, cudaStream_t st);
    std::string last_error;

private:
    int fail(const char* what, cudaError_t e);
    Engine eng_;
    DevBuf bKeys_, bCnt_, bCkpt_, bG_;
};

}  // namespace rdb
