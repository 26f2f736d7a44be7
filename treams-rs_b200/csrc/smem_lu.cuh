// Dense complex LU in shared memory by one CTA (all threads call these together): partial
// pivoting on the largest modulus (first index on ties, so results do not depend on the
// launch), and the solve of an M x nc right-hand-side panel against the factors.
#pragma once
#include "common.cuh"

namespace tcu {

constexpr int CTA_LU_MAXROWS = 3;  // rows per lane of the rank-1 update: M <= 96

// A: M x M column-major (shared, M <= 96), piv: M (shared), sing: one shared int set to 1 when a
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
        // rank-1 update: warps over columns, lanes over rows, the lane's multipliers in registers
        const int lane = tid & 31, warp = tid >> 5, nwarps = nth >> 5;
        cplx negl[CTA_LU_MAXROWS];
#pragma unroll
        for (int q = 0; q < CTA_LU_MAXROWS; ++q) {
            const int i = kc + 1 + lane + 32 * q;
            negl[q] = i < M ? cneg(A[kc * M + i]) : mk(0.0, 0.0);
        }
        for (int j = kc + 1 + warp; j < M; j += nwarps) {
            const cplx xk = A[j * M + kc];
#pragma unroll
            for (int q = 0; q < CTA_LU_MAXROWS; ++q) {
                const int i = kc + 1 + lane + 32 * q;
                if (i < M) {
                    cplx v = A[j * M + i];
                    cfma(v, negl[q], xk);
                    A[j * M + i] = v;
                }
            }
        }
        __syncthreads();
    }
    return true;
}

// B (M x nc column-major, shared) <- A^-1 B with the factors of cta_lu. One warp per
// right-hand side: the row interchanges, then forward and backward substitution with lanes
// over rows and only warp-level synchronisation between the steps. Every entry sees the same
// operations in the same order as a row-parallel sweep would apply them.
__device__ __forceinline__ void cta_lu_solve(const double2* A, int M, const int* piv, double2* B, int nc) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
    for (int jj = warp; jj < nc; jj += nwarps) {
        double2* b = B + jj * M;
        if (lane == 0)
            for (int kc = 0; kc < M; ++kc) {
                const int pr = piv[kc];
                if (pr != kc) {
                    double2 t = b[kc];
                    b[kc] = b[pr];
                    b[pr] = t;
                }
            }
        __syncwarp();
        for (int kc = 0; kc < M - 1; ++kc) {  // unit lower
            const cplx xk = b[kc];
            for (int i = kc + 1 + lane; i < M; i += 32) {
                cplx v = b[i];
                cfma(v, cneg(A[kc * M + i]), xk);
                b[i] = v;
            }
            __syncwarp();
        }
        for (int kc = M - 1; kc >= 0; --kc) {  // upper
            if (lane == 0) b[kc] = cmul(b[kc], cinv(A[kc * M + kc]));
            __syncwarp();
            const cplx xk = b[kc];
            for (int i = lane; i < kc; i += 32) {
                cplx v = b[i];
                cfma(v, cneg(A[kc * M + i]), xk);
                b[i] = v;
            }
            __syncwarp();
        }
    }
    __syncthreads();
}

}  // namespace tcu
