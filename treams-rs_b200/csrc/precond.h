// Right preconditioners of the matrix-free GMRES: block Jacobi over nearest-neighbour sphere
// groups (precond.cu) and the two-level coarse-dipole + near-field preconditioners, untrained
// or with a graph network's near-field weights (gnn.cu).
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

// Block Jacobi over nearest-neighbour sphere groups of at most 96 modes (precond.cu).
tcu_status make_block_jacobi(cudaStream_t st, const DevPlan& P, int N, double k0, const double* d_pos,
                             const double* h_pos, const double* h_radii, const double2* d_T,
                             std::unique_ptr<Preconditioner>* out, long long* launches);

bool tf32_enabled();

// Solves with the LU factor of a cluster's coarse (dipole) system, made by the API layer:
// v (6 N complex, device) <- A_cc^-1 v.
struct CoarseSolve {
    virtual ~CoarseSolve() {}
    virtual tcu_status solve(double2* v, cudaStream_t st) = 0;
};

// Two-level preconditioner (gnn.cu): coarse dipole correction, then the near field within
// reach sphere diameters with every (degree, degree) sub-block scaled by the graph network's
// Theta (learned, weights: the compiled-in weights of lmax when empty; without weights for
// lmax, Theta = 1) or by 1 (learned false: the untrained two-level method).
tcu_status make_two_level(cudaStream_t st, bool learned, const DevPlan& P, int L, int N, double k0,
                          const double* d_pos, const double* h_pos, const double* h_radii, const double* h_eps,
                          const double2* d_T, double reach, const std::vector<double>& weights,
                          std::unique_ptr<CoarseSolve> coarse, std::unique_ptr<Preconditioner>* out,
                          long long* launches);
int learned_weight_count(int L);

// One training cluster of the graph network: its graph, near-field blocks and coarse-corrected
// unit-norm probes r1 (from nprobe probe vectors V); loss_grad evaluates
// sum_p ||r1_p - A M_Theta r1_p||^2 and its gradient in every weight on the device.
class LearnedProblem {
   public:
    LearnedProblem();
    ~LearnedProblem();
    tcu_status build(cudaStream_t st, const DevPlan& P, int L, int N, double k0, const double* d_pos,
                     const double* h_pos, const double* h_radii, const double* h_eps, const double2* d_T, double reach,
                     int nprobe, const double2* d_V, std::unique_ptr<CoarseSolve> coarse, long long* launches);
    tcu_status loss_grad(const double* h_weights, double* loss, double* h_grad, cudaStream_t st);
    tcu_status probes(double2* h_out, cudaStream_t st);
    // y = (I - T C)^H x for ncol <= nprobe device columns (the adjoint operator of the loss)
    tcu_status adjoint_apply(const double2* d_x, double2* d_y, int ncol, cudaStream_t st);
    int L = 0, N = 0;
    double k0 = 0.0;
    size_t n = 0;
    const DevPlan* plan = nullptr;
    const double* d_pos = nullptr;
    const double2* d_T = nullptr;
    long long* launches = nullptr;
    struct Impl;
    std::unique_ptr<Impl> impl;
};

}  // namespace tcu
