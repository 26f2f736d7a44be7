// Right preconditioners of the matrix-free GMRES (block Jacobi over neighbour clusters and
// the learned block-sparse approximate inverse).
#pragma once
#include <cuda_runtime.h>

#include <memory>

#include "../../include/treams_cuda.h"
#include "plan.h"

namespace tcu {

class Preconditioner {
   public:
    virtual ~Preconditioner() {}
    // out = M in for one column of length n (device vectors, stream-ordered)
    virtual void apply(const double2* in, double2* out, cudaStream_t st) = 0;
};

tcu_status make_preconditioner(cudaStream_t st, int kind, const DevPlan& P, int L, int N, double k0,
                               const double* d_pos, const double2* d_T, std::unique_ptr<Preconditioner>* out,
                               long long* launches);

bool tf32_enabled();

}  // namespace tcu
