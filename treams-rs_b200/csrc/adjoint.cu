// Adjoint operator and adjoint LU solves of the cluster system (the pullbacks of
// cluster/interaction.rs:221-227 and cluster/iterative.rs:460-488).
//
// Matrix-free A^H: translation blocks satisfy the reciprocity C_ij[(lam,mu,t),(l,m,s)] =
// (-1)^(m+mu) C_ji[(l,-m,s),(lam,-mu,t)] (sw/plan.rs:725-800), i.e. C^T = F C F with the
// order flip (F x)(l, m, pol) = (-1)^m x(l, -m, pol), F = F^-1 real. Hence
//   A^H x = x - C^H T^H x = x - F conj(C conj(F T^H x)),
// one forward coupling product between two elementwise passes.
//
// Adjoint LU solve: the factors hold R A C = P^T L U (row and column scales R, C, real), so
// A^-H g = R P^T L^-H U^-H C g. U^H is lower triangular with block row b equal to the
// conjugate transpose of block column b of U above the diagonal; L^H is unit upper with block
// row b the conjugate transpose of block column b of L below the diagonal. Each block step
// reads those columns (contiguous in column-major storage), one CTA per column of the block,
// then applies the conjugate transpose of the stored FP64 inverse of the diagonal block.
#include <cuda_runtime.h>

#include <algorithm>

#include "common.cuh"
#include "kernels.h"

namespace tcu {

namespace {

constexpr int AB = 64;      // diagonal block size of the stored inverses (solve.cu)
constexpr int AMAXC = 8;    // right-hand sides per sweep

__device__ __forceinline__ int lm_deg(int lm) {  // lm = l*l - 1 + l + m
    int l = (int)sqrt((double)(lm + 1));
    while (l * l > lm + 1) --l;
    while ((l + 1) * (l + 1) <= lm + 1) ++l;
    return l;
}

// y = T^H x per sphere and degree (2 x 2 blocks in mode order, row-major)
__global__ void th_apply_kernel(int N, int L, const cplx* __restrict__ T, const cplx* __restrict__ x, size_t ldx,
                                int ncol, cplx* __restrict__ y) {
    const int nlm = L * (L + 2);
    const size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (size_t)N * nlm * ncol) return;
    const int c = (int)(t / ((size_t)N * nlm));
    const size_t r = t - (size_t)c * N * nlm;
    const int i = (int)(r / nlm), lm = (int)(r % nlm);
    const cplx* t4 = T + ((size_t)i * L + lm_deg(lm) - 1) * 4;
    const size_t o = c * ldx + (size_t)i * 2 * nlm + 2 * lm;
    const cplx a = x[o], b = x[o + 1];
    cplx y0 = mk(0.0, 0.0), y1 = mk(0.0, 0.0);
    cfma_conj(y0, t4[0], a);
    cfma_conj(y0, t4[2], b);
    cfma_conj(y1, t4[1], a);
    cfma_conj(y1, t4[3], b);
    y[o] = y0;
    y[o + 1] = y1;
}

// y = base - conj(F x) (base null: y = conj(F x))
__global__ void flip_conj_kernel(int N, int L, const cplx* __restrict__ x, const cplx* __restrict__ base, size_t ldx,
                                 int ncol, cplx* __restrict__ y) {
    const int M = 2 * L * (L + 2);
    const size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (size_t)N * M * ncol) return;
    const int c = (int)(t / ((size_t)N * M));
    const size_t r = t - (size_t)c * N * M;
    const int i = (int)(r / M), q = (int)(r % M);
    const int lm = q >> 1, slot = q & 1, l = lm_deg(lm), m = lm + 1 - l * l - l;
    const int src = 2 * (l * l - 1 + l - m) + slot;
    cplx v = cconj(x[c * ldx + (size_t)i * M + src]);
    if (m & 1) v = cneg(v);
    const size_t o = c * ldx + r;
    y[o] = base ? csub(base[o], v) : v;
}

// Block step of an adjoint sweep, part 1: CTA k forms t[c][k] = rhs[c][b0 + k] -
// sum_{r in [r0, r1)} conj(A[r][b0 + k]) sol[c][r] for the ncol columns (fixed-order tree
// reduction inside the CTA).
template <typename C>
__global__ void __launch_bounds__(256) adj_dot_kernel(const C* __restrict__ A, size_t lda, size_t n, int b0, int bw,
                                                      int r0, int r1, const double2* __restrict__ rhs,
                                                      const double2* __restrict__ sol, int ncol,
                                                      double2* __restrict__ t) {
    __shared__ double2 red[AMAXC][256];
    const int k = blockIdx.x;
    if (k >= bw) return;
    const C* a = A + (size_t)(b0 + k) * lda;
    double2 acc[AMAXC];
#pragma unroll
    for (int c = 0; c < AMAXC; ++c) acc[c] = mk(0.0, 0.0);
    for (int r = r0 + threadIdx.x; r < r1; r += blockDim.x) {
        const C av = a[r];
        const double2 v = mk((double)av.x, (double)av.y);
#pragma unroll
        for (int c = 0; c < AMAXC; ++c)
            if (c < ncol) cfma_conj(acc[c], v, sol[c * n + r]);
    }
#pragma unroll
    for (int c = 0; c < AMAXC; ++c)
        if (c < ncol) red[c][threadIdx.x] = acc[c];
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s)
            for (int c = 0; c < ncol; ++c) red[c][threadIdx.x] = cadd(red[c][threadIdx.x], red[c][threadIdx.x + s]);
        __syncthreads();
    }
    if (threadIdx.x < ncol) {
        const int c = threadIdx.x;
        t[c * AB + k] = csub(rhs[c * n + b0 + k], red[c][0]);
    }
}

// part 2: sol[c][b0 + i] = sum_k conj(Dinv[k][i]) t[c][k]  (Dinv column-major 64 x 64)
__global__ void adj_diag_kernel(const double2* __restrict__ dinv, int b0, int bw, size_t n, int ncol,
                                const double2* __restrict__ t, double2* __restrict__ sol) {
    const int i = threadIdx.x % AB, c = threadIdx.x / AB;
    if (c >= ncol || i >= bw) return;
    double2 s = mk(0.0, 0.0);
    for (int k = 0; k < bw; ++k) cfma_conj(s, dinv[(size_t)i * AB + k], t[c * AB + k]);
    sol[c * n + b0 + i] = s;
}

__global__ void scatter_perm_kernel(const double2* __restrict__ z, double2* __restrict__ y, const int* __restrict__ perm,
                                    int n, int ncol) {
    const size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (size_t)n * ncol) return;
    const int c = (int)(t / n), i = (int)(t % n);
    y[(size_t)c * n + perm[i]] = z[t];
}

unsigned nblk(size_t count, int threads) { return (unsigned)((count + threads - 1) / threads); }

template <typename C>
void adjoint_solve_impl(const C* A, int n, const int* perm, const double2* inv, double2* x, double2* tmp, int ncol,
                        cudaStream_t st, long long* launches) {
    StageScope sc(ST_SOLVE, st);
    const int nb = (n + AB - 1) / AB;
    const double2* linv = inv;
    const double2* uinv = inv + (size_t)nb * AB * AB;
    for (int c0 = 0; c0 < ncol; c0 += AMAXC) {
        const int nc = std::min(AMAXC, ncol - c0);
        double2* g = x + (size_t)c0 * n;       // right-hand side, then the solution
        double2* w = tmp;                      // U^-H g
        double2* z = tmp + (size_t)n * nc;     // L^-H w
        double2* tb = tmp + (size_t)2 * n * nc;  // 64 x nc block scratch
        // U^H w = g: blocks ascending, block column b of U above the diagonal
        for (int b = 0; b < nb; ++b) {
            const int b0 = b * AB, bw = std::min(AB, n - b0);
            adj_dot_kernel<C><<<bw, 256, 0, st>>>(A, (size_t)n, (size_t)n, b0, bw, 0, b0, g, w, nc, tb);
            adj_diag_kernel<<<1, AB * nc, 0, st>>>(uinv + (size_t)b * AB * AB, b0, bw, (size_t)n, nc, tb, w);
        }
        // L^H z = w: blocks descending, block column b of L below the diagonal
        for (int b = nb - 1; b >= 0; --b) {
            const int b0 = b * AB, bw = std::min(AB, n - b0);
            adj_dot_kernel<C><<<bw, 256, 0, st>>>(A, (size_t)n, (size_t)n, b0, bw, b0 + bw, n, w, z, nc, tb);
            adj_diag_kernel<<<1, AB * nc, 0, st>>>(linv + (size_t)b * AB * AB, b0, bw, (size_t)n, nc, tb, z);
        }
        scatter_perm_kernel<<<nblk((size_t)n * nc, 256), 256, 0, st>>>(z, g, perm, n, nc);
        if (launches) *launches += 4 * nb + 1;
    }
}

}  // namespace

void launch_apply_adjoint(const DevPlan& P, int N, double k0, const double* pos, const cplx* T, const cplx* x,
                          size_t ldx, int ncol, cplx* y, cplx* t1, cplx* t2, cudaStream_t st, long long* launches,
                          const cplx* Z, cplx* Xf, int* status) {
    const int L = P.L, nlm = P.nlm;
    const size_t n = (size_t)N * 2 * nlm;
    th_apply_kernel<<<nblk((size_t)N * nlm * ncol, 256), 256, 0, st>>>(N, L, T, x, ldx, ncol, t1);
    flip_conj_kernel<<<nblk(n * ncol, 256), 256, 0, st>>>(N, L, t1, nullptr, ldx, ncol, t2);
    if (Z) {  // the coupling product from the stored pair tables (T null: C alone)
        launch_apply_stored(P, N, STORED_FULL, Z, nullptr, t2, ldx, ncol, nullptr, 0.0, 1.0, t1, Xf, status, st);
        if (launches) *launches += 2;
    } else {
        for (int c0 = 0; c0 < ncol; c0 += 8) {
            const int nc = std::min(8, ncol - c0);
            launch_apply(P, N, k0, pos, nullptr, t2 + (size_t)c0 * ldx, ldx, nc, nullptr, 0.0, 1.0, true,
                         t1 + (size_t)c0 * ldx, st);
        }
        if (launches) *launches += (ncol + 7) / 8;
    }
    flip_conj_kernel<<<nblk(n * ncol, 256), 256, 0, st>>>(N, L, t1, x, ldx, ncol, y);
    if (launches) *launches += 3;
}

void launch_apply_th(int L, int N, const cplx* T, const cplx* x, size_t ldx, int ncol, cplx* y, cudaStream_t st) {
    const int nlm = L * (L + 2);
    th_apply_kernel<<<nblk((size_t)N * nlm * ncol, 256), 256, 0, st>>>(N, L, T, x, ldx, ncol, y);
}

size_t adjoint_solve_tmp(int n, int ncol) { return (size_t)2 * n * std::min(ncol, AMAXC) + (size_t)AB * AMAXC; }

void lu_solve_adjoint_fp64(const double2* A, int n, const int* perm, const double2* inv, double2* x, double2* tmp,
                           int ncol, cudaStream_t st, long long* launches) {
    adjoint_solve_impl<double2>(A, n, perm, inv, x, tmp, ncol, st, launches);
}
void lu_solve_adjoint_fp32(const float2* A, int n, const int* perm, const double2* inv, double2* x, double2* tmp,
                           int ncol, cudaStream_t st, long long* launches) {
    adjoint_solve_impl<float2>(A, n, perm, inv, x, tmp, ncol, st, launches);
}

}  // namespace tcu
