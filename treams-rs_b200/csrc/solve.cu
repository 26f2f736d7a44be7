// Triangular solves with the LU factors (FP64 or FP32 storage, FP64 arithmetic).
//
// After a factorization the diagonal 64 x 64 blocks of L (unit lower) and U (upper) are
// inverted once, in FP64 (tri_block_inverse_kernel). A forward or backward sweep is then a
// chain of block steps, each one launch: every CTA forms x_b = D_b^-1 r_b (a dense 64 x 64
// product, no serial recurrence) and subtracts the block column times x_b from its share
// of the remaining rows (read once, coalesced along the column). The right-hand side is
// updated in place while the block solutions go to a separate array, so no CTA reads a
// row that another CTA writes in the same step.
//
// The default sweep is one persistent kernel per triangle instead (trsv_chain_kernel): CTA c
// takes the block rows c, c + G, ... in solve order and accumulates L_ij y_j over its
// dependencies in a fixed order, consuming each y_j as soon as the block's completion flag
// carries this launch's epoch (release/acquire, bounded waits), so a sweep costs the chain
// of diagonal steps plus one pass over the factor instead of one launch per block.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdlib>
#include <string>

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

// ---- persistent sweep ------------------------------------------------------------------
constexpr int CH_JB = 8;  // block solutions staged per batch

__device__ __forceinline__ unsigned ch_ld_acquire(const unsigned* p) {
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ unsigned long long ch_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}
__device__ __forceinline__ void ch_cp16(void* smem, const void* gmem) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"((unsigned)__cvta_generic_to_shared(smem)),
                 "l"(gmem)
                 : "memory");
}

// Bounded wait (4 s) for flag == epoch; false (and status 8) when it gives up.
__device__ bool ch_wait(const unsigned* flag, unsigned epoch, int* status) {
    if (ch_ld_acquire(flag) == epoch) return true;
    const unsigned long long t0 = ch_ns();
    unsigned spins = 0;
    while (ch_ld_acquire(flag) != epoch) {
        if ((++spins & 255u) == 0 && (*(volatile int*)status == 8 || ch_ns() - t0 > 4000000000ull)) {
            atomicExch(status, 8);
            return false;
        }
    }
    return true;
}

template <typename C>
__host__ __device__ constexpr size_t chain_smem_bytes(int nc) {
    return ((size_t)SB * SB + (size_t)CH_JB * nc * SB + 4 * (size_t)nc * SB + (size_t)nc * SB) * sizeof(double2);
}

// y = T^-1 b for the unit lower (LOWER) or upper triangle T of the factor, with the FP64
// inverses of its diagonal blocks. rhs: b (n x NC, read only); sol: y. Block row i (solve
// order t) forms s = b_i - sum_j T_ij y_j over its dependencies in solve order, then
// y_i = Dinv_i s, stores it and releases flags[i] = epoch.
template <typename C, bool LOWER, int NC>
__global__ void __launch_bounds__(256) trsv_chain_kernel(const C* __restrict__ A, size_t lda, int n, int nb,
                                                         const double2* __restrict__ dinv,
                                                         const double2* __restrict__ rhs, double2* __restrict__ sol,
                                                         unsigned* __restrict__ flags, unsigned epoch,
                                                         int* __restrict__ status) {
    extern __shared__ __align__(16) double2 ch_smem[];
    double2* dsm = ch_smem;                    // Dinv of the current block row, column-major 64 x 64
    double2* ys = dsm + SB * SB;               // [CH_JB][NC][SB] staged block solutions
    double2* part = ys + CH_JB * NC * SB;      // [4][NC][SB]
    double2* sb = part + 4 * NC * SB;          // [NC][SB] right-hand side block
    __shared__ int s_ready;
    const int tid = threadIdx.x, ir = tid % SB, q = tid / SB;
    auto blk = [&](int t) { return LOWER ? t : nb - 1 - t; };
    int ready = 0;  // solve-order blocks known to be complete
    for (int t = blockIdx.x; t < nb; t += gridDim.x) {
        const int bi = blk(t), r0 = bi * SB, bw = min(SB, n - r0);
        const bool has_row = ir < bw;
        const size_t row = (size_t)r0 + (has_row ? ir : 0);
        // the diagonal inverse and the right-hand side block arrive in the background
        const double2* dsrc = dinv + (size_t)bi * SB * SB;
        for (int idx = tid; idx < SB * SB; idx += blockDim.x) ch_cp16(&dsm[idx], &dsrc[idx]);
        for (int idx = tid; idx < NC * SB; idx += blockDim.x) {
            const int ii = idx % SB, c = idx / SB;
            if (ii < bw)
                ch_cp16(&sb[idx], &rhs[(size_t)c * n + r0 + ii]);
            else
                sb[idx] = make_double2(0.0, 0.0);
        }
        asm volatile("cp.async.commit_group;" ::: "memory");
        double2 acc[NC];
#pragma unroll
        for (int c = 0; c < NC; ++c) acc[c] = make_double2(0.0, 0.0);
        C cur[16];
        auto load_block = [&](int ts, C (&v)[16]) {
            const int c0 = blk(ts) * SB + q * 16;
#pragma unroll
            for (int u = 0; u < 16; ++u) {
                if (has_row && c0 + u < n)
                    v[u] = A[(size_t)(c0 + u) * lda + row];
                else {
                    v[u].x = 0;
                    v[u].y = 0;
                }
            }
        };
        if (t > 0) load_block(0, cur);
        int ts = 0;
        while (ts < t) {
            if (ready <= ts) {
                __syncthreads();  // s_ready of the previous wait has been read by every thread
                if (tid == 0) {
                    int rdy = -1;
                    if (ch_wait(&flags[blk(ts)], epoch, status)) {
                        rdy = ts + 1;
                        while (rdy < t && rdy < ts + CH_JB && ch_ld_acquire(&flags[blk(rdy)]) == epoch) ++rdy;
                    }
                    s_ready = rdy;
                }
                __syncthreads();
                ready = s_ready;
                if (ready < 0) {
                    asm volatile("cp.async.wait_all;" ::: "memory");
                    return;
                }
            }
            const int cnt = min(CH_JB, ready - ts);
            for (int idx = tid; idx < cnt * NC * SB; idx += blockDim.x) {
                const int ii = idx % SB, c = (idx / SB) % NC, jj = idx / (SB * NC);
                const int gi = blk(ts + jj) * SB + ii;
                ys[idx] = gi < n ? __ldcg(&sol[(size_t)c * n + gi]) : make_double2(0.0, 0.0);
            }
            __syncthreads();
            for (int jj = 0; jj < cnt; ++jj) {
                C nxt[16];
                const bool more = ts + jj + 1 < t;
                if (more) load_block(ts + jj + 1, nxt);
#pragma unroll
                for (int u = 0; u < 16; ++u) {
                    const double lr = cur[u].x, li = cur[u].y;
#pragma unroll
                    for (int c = 0; c < NC; ++c) {
                        const double2 y = ys[(jj * NC + c) * SB + q * 16 + u];
                        acc[c].x += lr * y.x - li * y.y;
                        acc[c].y += lr * y.y + li * y.x;
                    }
                }
                if (more)
#pragma unroll
                    for (int u = 0; u < 16; ++u) cur[u] = nxt[u];
            }
            ts += cnt;
            __syncthreads();  // ys is restaged by the next batch
        }
#pragma unroll
        for (int c = 0; c < NC; ++c) part[(q * NC + c) * SB + ir] = acc[c];
        asm volatile("cp.async.wait_all;" ::: "memory");
        __syncthreads();
        for (int idx = tid; idx < NC * SB; idx += blockDim.x) {
            const int ii = idx % SB, c = idx / SB;
            double2 v = sb[idx];
#pragma unroll
            for (int qq = 0; qq < 4; ++qq) {
                v.x -= part[(qq * NC + c) * SB + ii].x;
                v.y -= part[(qq * NC + c) * SB + ii].y;
            }
            sb[idx] = v;
        }
        __syncthreads();
#pragma unroll
        for (int c = 0; c < NC; ++c) {
            double2 y = make_double2(0.0, 0.0);
#pragma unroll
            for (int u = 0; u < 16; ++u) {
                const double2 d = dsm[(q * 16 + u) * SB + ir], v = sb[c * SB + q * 16 + u];
                y.x += d.x * v.x - d.y * v.y;
                y.y += d.x * v.y + d.y * v.x;
            }
            part[(q * NC + c) * SB + ir] = y;
        }
        __syncthreads();
        for (int idx = tid; idx < NC * SB; idx += blockDim.x) {
            const int ii = idx % SB, c = idx / SB;
            if (ii < bw) {
                double2 y = part[c * SB + ii];
#pragma unroll
                for (int qq = 1; qq < 4; ++qq) {
                    y.x += part[(qq * NC + c) * SB + ii].x;
                    y.y += part[(qq * NC + c) * SB + ii].y;
                }
                sol[(size_t)c * n + r0 + ii] = y;
            }
        }
        __syncthreads();
        if (tid == 0) {
            __threadfence();
            asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(&flags[bi]), "r"(epoch) : "memory");
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

// the two sets of block inverses, then one completion flag per block (persistent sweeps)
size_t lu_inverse_bytes(int n) {
    const size_t nb = (n + SB - 1) / SB;
    return (size_t)2 * nb * SB * SB * sizeof(double2) + (nb + 64) * sizeof(unsigned);
}
static unsigned* chain_flags(const double2* inv, int n) {
    const size_t nb = (n + SB - 1) / SB;
    return (unsigned*)(inv + 2 * nb * SB * SB);
}

template <typename C>
static void inverses_impl(const C* A, int n, double2* inv, cudaStream_t st, long long* launches) {
    int nb = (n + SB - 1) / SB;
    StageScope sc(ST_SOLVE, st);
    const size_t smem = (size_t)(SB * (SB + 1) + SB) * sizeof(double2);
    static PerDeviceOnce attr;
    once_per_device(attr, [&] {
        cudaFuncSetAttribute(tri_block_inverse_kernel<double2, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        cudaFuncSetAttribute(tri_block_inverse_kernel<double2, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        cudaFuncSetAttribute(tri_block_inverse_kernel<float2, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        cudaFuncSetAttribute(tri_block_inverse_kernel<float2, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    });
    cudaMemsetAsync(chain_flags(inv, n), 0, (size_t)(nb + 64) * sizeof(unsigned), st);
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

// Persistent sweeps unless TCU_SOLVE=steps asks for one launch per block step.
static bool chain_enabled() {
    static const bool v = [] {
        const char* e = getenv("TCU_SOLVE");
        return !(e && std::string(e) == "steps");
    }();
    return v;
}

template <typename C, bool LOWER, int NC>
static bool chain_launch_nc(cudaStream_t st, const C* A, int n, const double2* dinv, const double2* rhs,
                            double2* sol, unsigned* flags, unsigned epoch, int* status) {
    static PerDeviceOnce attr;
    const size_t smem = chain_smem_bytes<C>(NC);
    // a refused attribute makes the cooperative launch below fail, and the caller takes the step path
    once_per_device(attr, [&] {
        cudaFuncSetAttribute(trsv_chain_kernel<C, LOWER, NC>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    });
    const int nb = (n + SB - 1) / SB;
    const int grid = std::min(nb, g_sms);
    size_t lda = (size_t)n;
    void* args[] = {(void*)&A, &lda, &n, (void*)&nb, (void*)&dinv, (void*)&rhs, &sol, &flags, &epoch, &status};
    return cudaLaunchCooperativeKernel((void*)trsv_chain_kernel<C, LOWER, NC>, dim3(grid), dim3(256), args, smem,
                                       st) == cudaSuccess;
}

template <typename C, bool LOWER>
static bool chain_launch(int nc, cudaStream_t st, const C* A, int n, const double2* dinv, const double2* rhs,
                         double2* sol, unsigned* flags, unsigned epoch, int* status) {
    switch (nc) {
#define CH_CASE(K) \
    case K: return chain_launch_nc<C, LOWER, K>(st, A, n, dinv, rhs, sol, flags, epoch, status);
        CH_CASE(1) CH_CASE(2) CH_CASE(3) CH_CASE(4) CH_CASE(5) CH_CASE(6) CH_CASE(7) CH_CASE(8)
#undef CH_CASE
    }
    return false;
}

// x (n x ncol) <- A^-1 x; tmp holds 2 n ncol complex.
template <typename C>
static void solve_impl(const C* A, int n, const int* perm, const double2* inv, double2* x, double2* tmp, int ncol,
                       cudaStream_t st, long long* launches, unsigned* epoch, int* status) {
    static PerDeviceOnce sms_once;
    once_per_device(sms_once, [] {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&g_sms, cudaDevAttrMultiProcessorCount, dev);
    });
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
        if (chain_enabled() && epoch && status) {
            // forward sweep y -> z, backward sweep z -> x; each launch has its own epoch
            unsigned* flags = chain_flags(inv, n);
            if (chain_launch<C, true>(nc, st, A, n, linv, y, z, flags, ++*epoch, status) &&
                chain_launch<C, false>(nc, st, A, n, uinv, z, xc, flags, ++*epoch, status)) {
                *launches += 2;
                continue;
            }
            // a launch that was refused leaves no work behind (the flags of later launches
            // carry new epochs); the step path below recomputes this column chunk
            cudaGetLastError();
            cudaMemsetAsync(z, 0, tot * sizeof(double2), st);
        }
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
                   cudaStream_t st, long long* launches, unsigned* epoch, int* status) {
    solve_impl<double2>(A, n, perm, inv, x, tmp, ncol, st, launches, epoch, status);
}
void lu_solve_fp32(const float2* A, int n, const int* perm, const double2* inv, double2* x, double2* tmp, int ncol,
                   cudaStream_t st, long long* launches, unsigned* epoch, int* status) {
    solve_impl<float2>(A, n, perm, inv, x, tmp, ncol, st, launches, epoch, status);
}

}  // namespace tcu
