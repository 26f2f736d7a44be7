// Dense complex LU in shared memory by one CTA (all threads call these together): partial
// pivoting on the largest modulus (first index on ties, so results do not depend on the
// launch), and the solve of an M x nc right-hand-side panel against the factors.
#pragma once
#include "common.cuh"

namespace tcu {

// A: M x M column-major (shared), piv: M (shared), sing: one shared int set to 1 when a
// pivot is exactly zero. Returns false (on every thread) for a singular matrix.
__device__ __forceinline__ bool cta_lu(double2* A, int M, int* piv, int* sing) {
    const int tid = threadIdx.x, nth = blockDim.x;
    if (tid == 0) *sing = 0;
    __syncthreads();
    for (int kc = 0; kc < M; ++kc) {
        if (tid < 32) {
            double best = -1.0;
            int bi = kc;
            for (int i = kc + tid; i < M; i += 32) {
                double v = cabs2(A[kc * M + i]);
                if (v > best) {
                    best = v;
                    bi = i;
                }
            }
            for (int off = 16; off > 0; off >>= 1) {
                double ov = __shfl_down_sync(0xffffffffu, best, off);
                int oi = __shfl_down_sync(0xffffffffu, bi, off);
                if (ov > best || (ov == best && oi < bi)) {
                    best = ov;
                    bi = oi;
                }
            }
            if (tid == 0) {
                piv[kc] = bi;
                if (!(best > 0.0)) *sing = 1;
            }
        }
        __syncthreads();
        const int pr = piv[kc];
        if (pr != kc)
            for (int j = tid; j < M; j += nth) {
                double2 t = A[j * M + kc];
                A[j * M + kc] = A[j * M + pr];
                A[j * M + pr] = t;
            }
        __syncthreads();
        if (*sing) return false;
        const cplx inv = cinv(A[kc * M + kc]);
        for (int i = kc + 1 + tid; i < M; i += nth) A[kc * M + i] = cmul(A[kc * M + i], inv);
        __syncthreads();
        const int rem = M - kc - 1;
        for (int it = tid; it < rem * rem; it += nth) {
            int j = kc + 1 + it / rem, i = kc + 1 + it % rem;
            cplx v = A[j * M + i];
            cfma(v, cneg(A[kc * M + i]), A[j * M + kc]);
            A[j * M + i] = v;
        }
        __syncthreads();
    }
    return true;
}

// B (M x nc column-major, shared) <- A^-1 B with the factors of cta_lu
__device__ __forceinline__ void cta_lu_solve(const double2* A, int M, const int* piv, double2* B, int nc) {
    const int tid = threadIdx.x, nth = blockDim.x;
    for (int kc = 0; kc < M; ++kc) {  // row interchanges in factorization order
        const int pr = piv[kc];
        if (pr != kc)
            for (int jj = tid; jj < nc; jj += nth) {
                double2 t = B[jj * M + kc];
                B[jj * M + kc] = B[jj * M + pr];
                B[jj * M + pr] = t;
            }
        __syncthreads();
    }
    for (int kc = 0; kc < M - 1; ++kc) {  // unit lower
        const int rem = M - kc - 1;
        for (int it = tid; it < rem * nc; it += nth) {
            int jj = it / rem, i = kc + 1 + it % rem;
            cplx v = B[jj * M + i];
            cfma(v, cneg(A[kc * M + i]), B[jj * M + kc]);
            B[jj * M + i] = v;
        }
        __syncthreads();
    }
    for (int kc = M - 1; kc >= 0; --kc) {  // upper
        const cplx inv = cinv(A[kc * M + kc]);
        for (int jj = tid; jj < nc; jj += nth) B[jj * M + kc] = cmul(B[jj * M + kc], inv);
        __syncthreads();
        for (int it = tid; it < kc * nc; it += nth) {
            int jj = it / kc, i = it % kc;
            cplx v = B[jj * M + i];
            cfma(v, cneg(A[kc * M + i]), B[jj * M + kc]);
            B[jj * M + i] = v;
        }
        __syncthreads();
    }
}

}  // namespace tcu
