// Triangular solves with the LU factors (FP64 or FP32 storage, FP64 arithmetic).
//
// After a factorization the diagonal 64 x 64 blocks of L (unit lower) and U (upper) are
// inverted once, in FP64 (tri_block_inverse_kernel). A forward or backward sweep is then a
// chain of block steps, each one launch: every CTA forms x_b = D_b^-1 r_b (a dense 64 x 64
// product, no serial recurrence) and subtracts the block column times x_b from its share
// of the remaining rows (read once, coalesced along the column). The right-hand side is
// updated in place while the block solutions go to a separate array, so no CTA reads a
// row that another CTA writes in the same step.
#include <cuda_runtime.h>

#include <algorithm>

#include "common.cuh"
#include "kernels.h"

namespace tcu {

constexpr int SB = 64;      // diagonal block size
constexpr int SMAXC = 8;    // right-hand sides per sweep

template <typename C>
__device__ __forceinline__ double2 to_d2(C v) {
    return make_double2((double)v.x, (double)v.y);
}

// One CTA per diagonal block: invert in place in shared memory (FP64), column by column.
// Lower (unit): columns right to left, X[i][j] = -sum_{k=j+1..i} X[i][k] L[k][j].
// Upper: columns left to right, X[j][j] = 1/U[j][j], X[i][j] = -sum_{k=i..j-1} X[i][k] U[k][j] X[j][j].
// Out: column-major 64 x 64 per block (identity beyond the matrix edge).
template <typename C, bool LOWER>
__global__ void __launch_bounds__(256) tri_block_inverse_kernel(const C* __restrict__ A, size_t lda, int n,
                                                                double2* __restrict__ out) {
    extern __shared__ double2 tbi_smem[];
    double2 (*M)[SB + 1] = (double2 (*)[SB + 1])tbi_smem;  // M[i][k]
    double2* col = tbi_smem + SB * (SB + 1);
    const int b0 = blockIdx.x * SB, bw = min(SB, n - b0);
    for (int idx = threadIdx.x; idx < SB * SB; idx += blockDim.x) {
        int i = idx % SB, k = idx / SB;
        double2 v = (i < bw && k < bw) ? to_d2(A[(size_t)(b0 + k) * lda + b0 + i]) : make_double2(i == k ? 1.0 : 0.0, 0.0);
        M[i][k] = v;
    }
    __syncthreads();
    const int i = threadIdx.x;  // rows handled by threads 0..63
    if (LOWER) {
        if (i < SB) M[i][i] = make_double2(1.0, 0.0);
        for (int j = SB - 2; j >= 0; --j) {
            if (i < SB) col[i] = M[i][j];
            __syncthreads();
            if (i < SB && i > j) {
                double2 s = make_double2(0.0, 0.0);
                for (int k = j + 1; k <= i; ++k) {
                    double2 x = (k == i) ? make_double2(1.0, 0.0) : M[i][k];
                    double2 l = col[k];
                    s.x += x.x * l.x - x.y * l.y;
                    s.y += x.x * l.y + x.y * l.x;
                }
                M[i][j] = make_double2(-s.x, -s.y);
            }
            __syncthreads();
        }
        if (i < SB)
            for (int k = i + 1; k < SB; ++k) M[i][k] = make_double2(0.0, 0.0);
    } else {
        for (int j = 0; j < SB; ++j) {
            if (i < SB) col[i] = M[i][j];
            __syncthreads();
            double2 d = col[j];
            double den = d.x * d.x + d.y * d.y;
            double2 inv = make_double2(d.x / den, -d.y / den);
            if (i < SB && i < j) {
                double2 s = make_double2(0.0, 0.0);
                for (int k = i; k < j; ++k) {
                    double2 x = M[i][k], u = col[k];
                    s.x += x.x * u.x - x.y * u.y;
                    s.y += x.x * u.y + x.y * u.x;
                }
                M[i][j] = make_double2(-(s.x * inv.x - s.y * inv.y), -(s.x * inv.y + s.y * inv.x));
            } else if (i == j) {
                M[i][j] = inv;
            }
            __syncthreads();
        }
        if (i < SB)
            for (int k = 0; k < i; ++k) M[i][k] = make_double2(0.0, 0.0);
    }
    __syncthreads();
    double2* o = out + (size_t)blockIdx.x * SB * SB;
    for (int idx = threadIdx.x; idx < SB * SB; idx += blockDim.x) {
        int ii = idx % SB, k = idx / SB;
        o[idx] = M[ii][k];
    }
}

__global__ void gather_kernel(const double2* __restrict__ x, double2* __restrict__ y, const int* __restrict__ perm,
                              int n, int ncol) {
    size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (size_t)n * ncol) return;
    int c = (int)(t / n), i = (int)(t % n);
    y[t] = x[(size_t)c * n + perm[i]];
}

// One block step: sol_b = Dinv_b r_b; r[other rows] -= A[other rows, block] sol_b.
// Every load that does not depend on the block solution (the Dinv quarter of each thread,
// the right-hand side block, the first half of the thread's row of the block column) is
// issued up front, so a step costs about two memory round trips.
template <typename C, bool LOWER, int NC>
__global__ void __launch_bounds__(256) trsv_inv_step_kernel(const C* __restrict__ A, size_t lda, int n, int b0, int bw,
                                                            const double2* __restrict__ dinv, double2* __restrict__ r,
                                                            double2* __restrict__ sol) {
    __shared__ double2 rb[NC][SB];
    __shared__ double2 part[4][NC][SB];
    __shared__ double2 xb[NC][SB];
    constexpr int KH = 16;  // preloaded first chunk of the block column
    // Programmatic dependent launch: the next step may start its read-only preloads (its
    // Dinv quarter and block column) while this one runs; it reads the right-hand side only
    // after griddepcontrol.wait, i.e. after this grid has completed and its writes are visible.
    asm volatile("griddepcontrol.launch_dependents;");
    const int tid = threadIdx.x;
    const int i = tid % SB, kq = tid / SB;  // Dinv row and K quarter
    double2 d[16];
#pragma unroll
    for (int u = 0; u < 16; ++u) d[u] = dinv[(size_t)(kq * 16 + u) * SB + i];
    const int lo = LOWER ? b0 + bw : 0, hi = LOWER ? n : b0;
    const int row = lo + blockIdx.x * blockDim.x + tid;
    const bool has_row = row < hi;
    C av[KH];
#pragma unroll
    for (int u = 0; u < KH; ++u) {
        if (has_row && u < bw)
            av[u] = A[(size_t)(b0 + u) * lda + row];
        else {
            av[u].x = 0;
            av[u].y = 0;
        }
    }
    asm volatile("griddepcontrol.wait;" ::: "memory");
    for (int idx = tid; idx < SB * NC; idx += blockDim.x) {
        int ii = idx % SB, c = idx / SB;
        rb[c][ii] = ii < bw ? r[(size_t)c * n + b0 + ii] : make_double2(0.0, 0.0);
    }
    __syncthreads();
#pragma unroll
    for (int c = 0; c < NC; ++c) {
        double2 acc = make_double2(0.0, 0.0);
#pragma unroll
        for (int u = 0; u < 16; ++u) {
            double2 v = rb[c][kq * 16 + u];
            acc.x += d[u].x * v.x - d[u].y * v.y;
            acc.y += d[u].x * v.y + d[u].y * v.x;
        }
        part[kq][c][i] = acc;
    }
    __syncthreads();
    for (int idx = tid; idx < SB * NC; idx += blockDim.x) {
        int ii = idx % SB, c = idx / SB;
        double2 s = part[0][c][ii];
#pragma unroll
        for (int q = 1; q < 4; ++q) {
            s.x += part[q][c][ii].x;
            s.y += part[q][c][ii].y;
        }
        xb[c][ii] = s;
    }
    __syncthreads();
    if (blockIdx.x == 0)
        for (int idx = tid; idx < bw * NC; idx += blockDim.x) {
            int ii = idx % bw, c = idx / bw;
            sol[(size_t)c * n + b0 + ii] = xb[c][ii];
        }
    // rows beyond the first pass of the grid (n > 148 * 256) load their first chunk here too
    for (int rr = row; rr < hi; rr += gridDim.x * blockDim.x) {
        const bool first = rr == row;
        double2 acc[NC];
#pragma unroll
        for (int c = 0; c < NC; ++c) acc[c] = make_double2(0, 0);
#pragma unroll 1
        for (int kc = 0; kc < SB; kc += KH) {
            C v[KH];
#pragma unroll
            for (int u = 0; u < KH; ++u) {
                if (kc == 0 && first)
                    v[u] = av[u];
                else if (kc + u < bw)
                    v[u] = A[(size_t)(b0 + kc + u) * lda + rr];
                else {
                    v[u].x = 0;
                    v[u].y = 0;
                }
            }
#pragma unroll
            for (int u = 0; u < KH; ++u) {
                double lr = v[u].x, li = v[u].y;
#pragma unroll
                for (int c = 0; c < NC; ++c) {
                    double2 x = xb[c][kc + u];
                    acc[c].x += lr * x.x - li * x.y;
                    acc[c].y += lr * x.y + li * x.x;
                }
            }
        }
#pragma unroll
        for (int c = 0; c < NC; ++c) {
            double2* p = r + (size_t)c * n + rr;
            double2 v = *p;
            v.x -= acc[c].x;
            v.y -= acc[c].y;
            *p = v;
        }
    }
}

static int g_sms = 0;

template <typename C, bool LOWER, int NC>
static void step_launch_nc(cudaStream_t st, const C* A, int n, int b0, int bw, const double2* dinv, double2* r,
                           double2* sol) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(g_sms);
    cfg.blockDim = dim3(256);
    cfg.dynamicSmemBytes = 0;
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    cudaLaunchKernelEx(&cfg, trsv_inv_step_kernel<C, LOWER, NC>, A, (size_t)n, n, b0, bw, dinv, r, sol);
}

template <typename C, bool LOWER>
static void step_launch(int nc, cudaStream_t st, const C* A, int n, int b0, int bw, const double2* dinv, double2* r,
                        double2* sol) {
    switch (nc) {
#define TV_CASE(K) \
    case K: step_launch_nc<C, LOWER, K>(st, A, n, b0, bw, dinv, r, sol); break;
        TV_CASE(1) TV_CASE(2) TV_CASE(3) TV_CASE(4) TV_CASE(5) TV_CASE(6) TV_CASE(7) TV_CASE(8)
#undef TV_CASE
    }
}

size_t lu_inverse_bytes(int n) { return (size_t)2 * ((n + SB - 1) / SB) * SB * SB * sizeof(double2); }

template <typename C>
static void inverses_impl(const C* A, int n, double2* inv, cudaStream_t st, long long* launches) {
    int nb = (n + SB - 1) / SB;
    StageScope sc(ST_SOLVE, st);
    const size_t smem = (size_t)(SB * (SB + 1) + SB) * sizeof(double2);
    static bool attr = false;
    if (!attr) {
        cudaFuncSetAttribute(tri_block_inverse_kernel<double2, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        cudaFuncSetAttribute(tri_block_inverse_kernel<double2, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        cudaFuncSetAttribute(tri_block_inverse_kernel<float2, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        cudaFuncSetAttribute(tri_block_inverse_kernel<float2, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        attr = true;
    }
    tri_block_inverse_kernel<C, true><<<nb, 256, smem, st>>>(A, n, n, inv);
    tri_block_inverse_kernel<C, false><<<nb, 256, smem, st>>>(A, n, n, inv + (size_t)nb * SB * SB);
    *launches += 2;
}
void lu_block_inverses_fp64(const double2* A, int n, double2* inv, cudaStream_t st, long long* launches) {
    inverses_impl<double2>(A, n, inv, st, launches);
}
void lu_block_inverses_fp32(const float2* A, int n, double2* inv, cudaStream_t st, long long* launches) {
    inverses_impl<float2>(A, n, inv, st, launches);
}

// x (n x ncol) <- A^-1 x; tmp holds 2 n ncol complex.
template <typename C>
static void solve_impl(const C* A, int n, const int* perm, const double2* inv, double2* x, double2* tmp, int ncol,
                       cudaStream_t st, long long* launches) {
    if (!g_sms) {
        int dev;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&g_sms, cudaDevAttrMultiProcessorCount, dev);
    }
    StageScope sc(ST_SOLVE, st);
    const int nb = (n + SB - 1) / SB;
    const double2* linv = inv;
    const double2* uinv = inv + (size_t)nb * SB * SB;
    for (int c0 = 0; c0 < ncol; c0 += SMAXC) {
        int nc = std::min(SMAXC, ncol - c0);
        double2* xc = x + (size_t)c0 * n;
        double2* y = tmp;                  // P b, then updated in place by the forward sweep
        double2* z = tmp + (size_t)n * nc; // forward solution, updated in place by the backward sweep
        size_t tot = (size_t)n * nc;
        gather_kernel<<<(unsigned)((tot + 255) / 256), 256, 0, st>>>(xc, y, perm, n, nc);
        ++*launches;
        for (int b = 0; b < nb; ++b) {
            int b0 = b * SB, bw = std::min(SB, n - b0);
            step_launch<C, true>(nc, st, A, n, b0, bw, linv + (size_t)b * SB * SB, y, z);
            ++*launches;
        }
        for (int b = nb - 1; b >= 0; --b) {
            int b0 = b * SB, bw = std::min(SB, n - b0);
            step_launch<C, false>(nc, st, A, n, b0, bw, uinv + (size_t)b * SB * SB, z, xc);
            ++*launches;
        }
    }
}

void lu_solve_fp64(const double2* A, int n, const int* perm, const double2* inv, double2* x, double2* tmp, int ncol,
                   cudaStream_t st, long long* launches) {
    solve_impl<double2>(A, n, perm, inv, x, tmp, ncol, st, launches);
}
void lu_solve_fp32(const float2* A, int n, const int* perm, const double2* inv, double2* x, double2* tmp, int ncol,
                   cudaStream_t st, long long* launches) {
    solve_impl<float2>(A, n, perm, inv, x, tmp, ncol, st, launches);
}

}  // namespace tcu
