// Right preconditioners of the matrix-free GMRES (block Jacobi over nearest-neighbour sphere
// groups, and the learned polynomial in the block-sparse near-field couplings).
#pragma once
#include <cuda_runtime.h>

#include <complex>
#include <memory>
#include <vector>

#include "../../include/treams_cuda.h"
#include "plan.h"

namespace tcu {

class Preconditioner {
   public:
    virtual ~Preconditioner() {}
    // out = M in for one column of length n (device vectors, stream-ordered)
    virtual void apply(const double2* in, double2* out, cudaStream_t st) = 0;
};

// kind: TCU_PRECOND_BLOCK_JACOBI or TCU_PRECOND_LEARNED. Positions and radii are given on
// the device (d_pos) and on the host (h_pos, h_radii: neighbour lists and blocks).
// reach: near-field reach in sphere diameters; layers < 0 selects the compiled-in fit, else
// alpha (layers + 1 weights; empty: all 1) is used.
tcu_status make_preconditioner(cudaStream_t st, int kind, const DevPlan& P, int L, int N, double k0,
                               const double* d_pos, const double* h_pos, const double* h_radii, const double2* d_T,
                               double reach, int layers, const std::vector<std::complex<double>>& alpha,
                               std::unique_ptr<Preconditioner>* out, long long* launches);

// Gram matrix G[k][l] = sum_v conj(u_k) . u_l and right-hand side b[k] = sum_v conj(u_k) . v of
// the learned preconditioner's layer basis u_k = A (D N)^k D v over nvec device vectors V
// (n x nvec): ||v - sum_k alpha_k u_k||^2 summed over v = const - 2 Re(alpha^H b) + alpha^H G alpha.
tcu_status learned_gram(cudaStream_t st, const DevPlan& P, int L, int N, double k0, const double* d_pos,
                        const double* h_pos, const double* h_radii, const double2* d_T, double reach, int layers,
                        int nvec,
                        const double2* d_V, double2* d_gram_scratch, double2* d_partial, std::complex<double>* gram,
                        std::complex<double>* rhs, long long* launches);

bool tf32_enabled();

}  // namespace tcu
