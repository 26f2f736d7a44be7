// Dense right-looking blocked LU with partial pivoting of a complex n x n column-major
// matrix, FP64 (double2) or FP32 (float2) storage.
//
// Per panel of width w (64 complex columns in FP64, 128 in FP32):
//  1. panel_kernel (cooperative, one CTA per SM): every CTA holds a slab of the panel rows
//     in shared memory; per column one grid barrier publishes each CTA's pivot candidate
//     (largest |a|, ties to the lower row) with its row and the current diagonal row, so
//     every CTA picks the same pivot, swaps locally and applies the rank-1 update.
//  2. laswp_kernel: the panel's row swaps on the columns outside it (skips identities).
//  3. U12 = L11^-1 A12: trsm_kernel (FP64, one warp per column), or in the mixed path the
//     blocked inverse of L11 (tri_inverse_l_kernel) and a tensor-core GEMM (gemm_tf32.cu).
//  4. trailing update A22 -= L21 U12: FP64 DMMA (mma.sync m8n8k4 f64) complex GEMM, or in
//     the mixed path the 3-pass split tcgen05 GEMM of gemm_tf32.cu.
// The permutation is composed from the pivots afterwards; the triangular solves with the
// factors are in solve.cu.
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>
#include <cstdlib>
#include <map>
#include <string>

#include "common.cuh"
#include "kernels.h"

namespace tcu {

template <typename R>
struct Cx;
template <>
struct Cx<double> {
    typedef double2 T;
};
template <>
struct Cx<float> {
    typedef float2 T;
};

template <typename C>
__device__ __forceinline__ C cx_make(double r, double i);
template <>
__device__ __forceinline__ double2 cx_make<double2>(double r, double i) {
    return make_double2(r, i);
}
template <>
__device__ __forceinline__ float2 cx_make<float2>(double r, double i) {
    return make_float2((float)r, (float)i);
}

struct Cand {
    double val;
    int row;
    int pad;
};

__device__ __forceinline__ unsigned ld_acquire_u32(const unsigned* p) {
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ unsigned long long global_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

constexpr int PANEL_THREADS = 256;
constexpr int PANEL_SUB = 16;  // columns per sub-block of the blocked panel update  // measured: 512 threads per CTA were slower

template <typename R>
__device__ __forceinline__ double cx_abs2(typename Cx<R>::T a) {
    return (double)a.x * (double)a.x + (double)a.y * (double)a.y;
}

// ---- panel factorization ------------------------------------------------------------------
// Per column every CTA publishes its best local candidate row, folds its candidate key
//   [|a|^2 as FP32 bits : 32][0xFFFFFFFF - row : 32]
// into one 64-bit atomicMax word (three words cycle over the columns), and arrives at a grid
// barrier (fire-and-forget release add on a counter that only grows, acquire polls). After
// the barrier every CTA
// reads the winning key and the pivot row: the largest |a| with ties to the lower row.
// Grid barrier of the cooperative panel: thread 0 of each CTA arrives with a release add and
// spins on acquire loads (no sleep: the wait is one column's latency); bounded at 4 s, after
// which it records status 8 (TCU_TIMEOUT) and every CTA returns.
constexpr unsigned long long BARRIER_LIMIT_NS = 4000000000ull;
__device__ bool column_barrier(unsigned* bar, unsigned target, int* status,
                               unsigned long long limit_ns = BARRIER_LIMIT_NS) {
    __shared__ int s_ok;
    __syncthreads();
    if (threadIdx.x == 0) {
        int ok = 1;
        __threadfence();
        asm volatile("red.release.gpu.global.add.u32 [%0], 1;" ::"l"(bar) : "memory");
        if (ld_acquire_u32(bar) < target) {
            unsigned long long t0 = global_ns();
            unsigned spins = 0;
            while (ld_acquire_u32(bar) < target) {
                if ((++spins & 1023u) == 0) {
                    if (*(volatile int*)status == 8 || global_ns() - t0 > limit_ns) {
                        atomicExch(status, 8);
                        ok = 0;
                        break;
                    }
                }
            }
        }
        s_ok = ok;
    }
    __syncthreads();
    return s_ok != 0;
}

// Candidate keys inside a CTA: [FP32 bits of |a|^2, + 1 : 32] (0 = no candidate) and the
// global row; the maximum key wins, ties to the lower row (redux.sync on both words).
__device__ __forceinline__ void warp_argmax(unsigned& key, unsigned& row) {
    const unsigned m = __reduce_max_sync(0xffffffffu, key);
    row = __reduce_min_sync(0xffffffffu, key == m ? row : 0xFFFFFFFFu);
    key = m;
}

// SUB = 0: every column's rank-1 update spans the rest of the panel. SUB = 16: the rank-1
// updates stay inside 16-column sub-blocks; after the last column of a sub-block every CTA
// forms the sub-block's 16 rows of U over the remaining columns from the 16 broadcast pivot
// rows it kept (forward substitution with their multipliers) and applies one rank-16 update
// to its rows below, so the trailing part of the slab is read and written once per 16
// columns instead of once per column.
template <typename R, int NB, int SUB>
__global__ void __launch_bounds__(PANEL_THREADS) panel_kernel(typename Cx<R>::T* A, size_t lda, int k0, int n, int w,
                                                    int chunk, int* piv, int* perm, unsigned long long* keys,
                                                    typename Cx<R>::T* crow, typename Cx<R>::T* drow, unsigned* bar,
                                                    int* status) {
    typedef typename Cx<R>::T C;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    C* tile = (C*)smem_raw;                      // chunk x (NB + 1)
    C* pbuf = tile + (size_t)chunk * (NB + 1);   // max(SUB, 1) pivot rows of NB
    __shared__ unsigned s_key[PANEL_THREADS / 32];
    __shared__ unsigned s_row[PANEL_THREADS / 32];
    __shared__ double s_inv[2];
    const int P = gridDim.x, b = blockIdx.x, tid = threadIdx.x;
    const int lane = tid & 31, warp = tid >> 5;
    const int rows = n - k0;
    const int row0 = k0 + b * chunk;
    const int myrows = max(0, min(chunk, rows - b * chunk));
    const int LD = NB + 1;
    for (int idx = tid; idx < myrows * w; idx += blockDim.x) {
        int r = idx % myrows, c = idx / myrows;
        tile[(size_t)r * LD + c] = A[(size_t)(k0 + c) * lda + row0 + r];
    }
    __syncthreads();
    // candidate of this thread's rows for column 0
    unsigned bk = 0u, br = 0xFFFFFFFFu;
    auto offer = [&](C v, int g) {
        const unsigned k = __float_as_uint((float)cx_abs2<R>(v)) + 1u;
        if (k > bk || (k == bk && (unsigned)g < br)) {
            bk = k;
            br = (unsigned)g;
        }
    };
    for (int r = tid; r < myrows; r += blockDim.x) offer(tile[(size_t)r * LD], row0 + r);
    for (int j = 0; j < w; ++j) {
        const int gj = k0 + j;
        const int buf = j & 1;
        const int jb = SUB ? j - j % SUB : 0;
        const int cend = SUB ? min(w, jb + SUB) : w;  // rank-1 updates stop here
        C* prow = pbuf + (size_t)(SUB ? j - jb : 0) * NB;
        warp_argmax(bk, br);
        if (lane == 0) {
            s_key[warp] = bk;
            s_row[warp] = br;
        }
        __syncthreads();
        unsigned ck = lane < PANEL_THREADS / 32 ? s_key[lane] : 0u;
        unsigned crr = lane < PANEL_THREADS / 32 ? s_row[lane] : 0xFFFFFFFFu;
        warp_argmax(ck, crr);
        const bool has = ck != 0u;
        if (has) {
            int lr = (int)crr - row0;
            for (int c = tid; c < w; c += blockDim.x) __stcg(&crow[((size_t)buf * P + b) * NB + c], tile[(size_t)lr * LD + c]);
        }
        if (gj >= row0 && gj < row0 + myrows) {
            int lr = gj - row0;
            for (int c = tid; c < w; c += blockDim.x) __stcg(&drow[(size_t)buf * NB + c], tile[(size_t)lr * LD + c]);
        }
        if (tid == 0 && has) {
            unsigned long long kv = ((unsigned long long)(ck - 1u) << 32) | (unsigned long long)(0xFFFFFFFFu - crr);
            asm volatile("red.relaxed.gpu.global.max.u64 [%0], %1;" ::"l"(&keys[j % 3]), "l"(kv) : "memory");
        }
        if (!column_barrier(bar, (unsigned)(j + 1) * (unsigned)P, status)) return;
        // The winning key and, speculatively, the diagonal row in one round trip: when the
        // pivot is the diagonal row (no interchange) the pivot row is already here.
        const unsigned long long key = __ldcg(&keys[j % 3]);
        C dv;
        dv.x = 0;
        dv.y = 0;
        if (tid < w) dv = __ldcg(&drow[(size_t)buf * NB + tid]);
        if (b == 0 && tid == 0) {
            // the word of column j-1, read by every CTA before this barrier
            *(volatile unsigned long long*)&keys[(j + 2) % 3] = 0ull;
        }
        const int pr = (int)(0xFFFFFFFFu - (unsigned)(key & 0xFFFFFFFFull));
        const int owner = (pr - k0) / chunk;
        if (tid < w) prow[tid] = (pr == gj) ? dv : __ldcg(&crow[((size_t)buf * P + owner) * NB + tid]);
        __syncthreads();
        if (pr != gj) {
            if (pr >= row0 && pr < row0 + myrows) {
                int lr = pr - row0;
                if (tid < w) tile[(size_t)lr * LD + tid] = dv;
            }
            if (gj >= row0 && gj < row0 + myrows) {
                int lr = gj - row0;
                for (int c = tid; c < w; c += blockDim.x) tile[(size_t)lr * LD + c] = prow[c];
            }
        }
        if (tid == 0) {
            // 1 / pivot once per CTA, in FP64
            C pivot = prow[j];
            double den = (double)pivot.x * pivot.x + (double)pivot.y * pivot.y;
            s_inv[0] = den > 0.0 ? pivot.x / den : 0.0;
            s_inv[1] = den > 0.0 ? -pivot.y / den : 0.0;
            if (b == 0) {
                piv[gj] = pr;  // the row permutation is composed from piv after the factorization
                if (!(den > 0.0)) atomicCAS(status, 0, 5);
            }
        }
        __syncthreads();
        // rank-1 update of the rows below the pivot; each thread keeps its next candidate
        const double ir = s_inv[0], ii = s_inv[1];
        const bool nonzero = ir != 0.0 || ii != 0.0;
        bk = 0u;
        br = 0xFFFFFFFFu;
        const int first = max(0, gj + 1 - row0);  // first local row below the pivot
        const int act = myrows - first;
        if (act > 0) {
            // S threads per row (a power of two up to 8, adjacent lanes of one warp): each forms
            // the row's multiplier, part 0 stores it, and part p updates the column batches
            // p, p + S, ... of j+1..cend-1. A batch's loads are issued before its stores, so its
            // shared-memory round trips overlap (a per-element loop would serialise them on the
            // possible aliasing of the row and the pivot row).
            constexpr int BATCH = sizeof(R) == 4 ? 8 : 4;
            const int ncols = cend - j - 1;
            int S = 1;
            while (S < 8 && act * S * 2 <= (int)blockDim.x && BATCH * S < ncols) S *= 2;
            for (int base = 0; base < act * S; base += blockDim.x) {  // one pass when S > 1
                const int it = base + tid;
                const bool valid = it < act * S;
                const int r = first + (valid ? it / S : 0), part = it % S;
                C* trow = tile + (size_t)r * LD;
                C a = trow[j];
                if (S > 1) __syncwarp();  // every part has read a before part 0 overwrites it
                C l;
                l.x = (R)(a.x * ir - a.y * ii);
                l.y = (R)(a.x * ii + a.y * ir);
                if (valid && part == 0 && nonzero) trow[j] = l;
                if (!valid) continue;
                for (int c = j + 1 + part * BATCH; c < cend; c += BATCH * S) {
                    C u[BATCH], t[BATCH];
#pragma unroll
                    for (int k = 0; k < BATCH; ++k)
                        if (c + k < cend) {
                            u[k] = prow[c + k];
                            t[k] = trow[c + k];
                        }
                    if (nonzero) {
#pragma unroll
                        for (int k = 0; k < BATCH; ++k)
                            if (c + k < cend) {
                                t[k].x = t[k].x - (l.x * u[k].x - l.y * u[k].y);
                                t[k].y = t[k].y - (l.x * u[k].y + l.y * u[k].x);
                                trow[c + k] = t[k];
                            }
                    }
                    if (c == j + 1) offer(t[0], row0 + r);
                }
            }
        }
        if (SUB && j + 1 == cend && cend < w) {
            // end of a full sub-block: U rows of its pivots over columns cend..w-1 (forward
            // substitution on the kept pivot rows, in place), then the rank-SUB update of the
            // rows below, which also yields the candidates of column cend.
            constexpr int SB = SUB ? SUB : 1;
            __syncthreads();
            for (int c = cend + tid; c < w; c += blockDim.x) {
                C u[SB];
#pragma unroll
                for (int k = 0; k < SB; ++k) {
                    C acc = pbuf[(size_t)k * NB + c];
#pragma unroll
                    for (int i = 0; i < k; ++i) {
                        const C lki = pbuf[(size_t)k * NB + jb + i];
                        acc.x = acc.x - (lki.x * u[i].x - lki.y * u[i].y);
                        acc.y = acc.y - (lki.x * u[i].y + lki.y * u[i].x);
                    }
                    u[k] = acc;
                    pbuf[(size_t)k * NB + c] = acc;
                }
            }
            __syncthreads();
            const int nt = w - cend;
            for (int idx = tid; idx < SB * nt; idx += blockDim.x) {
                const int k = idx / nt, c = cend + idx % nt, pos = k0 + jb + k;
                if (pos >= row0 && pos < row0 + myrows) tile[(size_t)(pos - row0) * LD + c] = pbuf[(size_t)k * NB + c];
            }
            constexpr int G = sizeof(R) == 4 ? 8 : 4;  // columns per item
            const int fc = max(0, k0 + cend - row0), ac = myrows - fc, ng = (nt + G - 1) / G;
            for (int item = tid; item < ac * ng; item += blockDim.x) {
                const int r = fc + item % ac, c0 = cend + (item / ac) * G;
                C* trow = tile + (size_t)r * LD;
                C acc[G];
#pragma unroll
                for (int k = 0; k < G; ++k)
                    if (c0 + k < w) acc[k] = trow[c0 + k];
#pragma unroll 4
                for (int i = 0; i < SB; ++i) {
                    const C li = trow[jb + i];
#pragma unroll
                    for (int k = 0; k < G; ++k)
                        if (c0 + k < w) {
                            const C u = pbuf[(size_t)i * NB + c0 + k];
                            acc[k].x = acc[k].x - (li.x * u.x - li.y * u.y);
                            acc[k].y = acc[k].y - (li.x * u.y + li.y * u.x);
                        }
                }
#pragma unroll
                for (int k = 0; k < G; ++k)
                    if (c0 + k < w) trow[c0 + k] = acc[k];
                if (c0 == cend) offer(acc[0], row0 + r);
            }
        }
        __syncthreads();
    }
    for (int idx = tid; idx < myrows * w; idx += blockDim.x) {
        int r = idx % myrows, c = idx / myrows;
        A[(size_t)(k0 + c) * lda + row0 + r] = tile[(size_t)r * LD + c];
    }
}

// ---- row swaps outside the panel ------------------------------------------------------------
template <typename C>
__global__ void laswp_kernel(C* A, size_t lda, int n, int k0, int w, const int* __restrict__ piv) {
    __shared__ int sp[128];
    __shared__ int any;
    if (threadIdx.x == 0) any = 0;
    __syncthreads();
    for (int j = threadIdx.x; j < w; j += blockDim.x) {
        sp[j] = piv[k0 + j];
        if (sp[j] != k0 + j) any = 1;
    }
    __syncthreads();
    if (!any) return;
    int col = blockIdx.x * blockDim.x + threadIdx.x;
    if (col >= n || (col >= k0 && col < k0 + w)) return;
    C* a = A + (size_t)col * lda;
    for (int j = 0; j < w; ++j) {
        int p = sp[j];
        if (p != k0 + j) {
            C t = a[k0 + j];
            a[k0 + j] = a[p];
            a[p] = t;
        }
    }
}

// ---- U12 = L11^-1 A12 ---------------------------------------------------------------------
template <typename R, int NB>
__global__ void __launch_bounds__(256) trsm_kernel(typename Cx<R>::T* A, size_t lda, int k0, int w, int n,
                                                   int cols_per_cta) {
    typedef typename Cx<R>::T C;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    C* Ls = (C*)smem_raw;  // Ls[k * NB + i] = L[i][k]
    for (int idx = threadIdx.x; idx < w * w; idx += blockDim.x) {
        int i = idx % w, k = idx / w;
        Ls[k * NB + i] = A[(size_t)(k0 + k) * lda + k0 + i];
    }
    __syncthreads();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    constexpr int S = NB / 32;
    int cbeg = k0 + w + blockIdx.x * cols_per_cta;
    int cend = min(n, cbeg + cols_per_cta);
    for (int col = cbeg + warp; col < cend; col += blockDim.x >> 5) {
        C* a = A + (size_t)col * lda + k0;
        R xr[S], xi[S];
#pragma unroll
        for (int s = 0; s < S; ++s) {
            int i = lane + 32 * s;
            C v = (i < w) ? a[i] : cx_make<C>(0.0, 0.0);
            xr[s] = v.x;
            xi[s] = v.y;
        }
#pragma unroll
        for (int kb = 0; kb < S; ++kb) {
            for (int kk = 0; kk < 32; ++kk) {
                int k = kb * 32 + kk;
                if (k >= w) break;
                R br = __shfl_sync(0xffffffffu, xr[kb], kk);
                R bi = __shfl_sync(0xffffffffu, xi[kb], kk);
#pragma unroll
                for (int s = kb; s < S; ++s) {
                    int i = lane + 32 * s;
                    if (i > k && i < w) {
                        C l = Ls[k * NB + i];
                        xr[s] -= l.x * br - l.y * bi;
                        xi[s] -= l.x * bi + l.y * br;
                    }
                }
            }
        }
#pragma unroll
        for (int s = 0; s < S; ++s) {
            int i = lane + 32 * s;
            if (i < w) {
                C v;
                v.x = xr[s];
                v.y = xi[s];
                a[i] = v;
            }
        }
    }
}

// ---- FP64 complex GEMM on DMMA: A22 -= L21 U12 -------------------------------------------
// CTA tile 64 x 64 complex; K = w complex in chunks of 16 staged by cp.async (2 stages).
// The complex product runs as a real GEMM of the 2x2-embedded L21 (rows re/im interleaved)
// with U12 read as interleaved reals: D[2mu+c][nu] = sum_k Lemb[2mu+c][2k+c'] U[2k+c'][nu].
__device__ __forceinline__ void cp_async16(void* smem, const void* gmem, bool valid) {
    unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    int sz = valid ? 16 : 0;
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(s), "l"(gmem), "r"(sz) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
    asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

constexpr int ZG_T = 64;   // tile rows/cols (complex)
constexpr int ZG_KC = 16;  // K chunk (complex)
constexpr size_t ZG_SMEM = 4 * ZG_KC * ZG_T * sizeof(double2);

__global__ void __launch_bounds__(256, 2) zgemm_dmma_kernel(double2* A, size_t lda, int k0, int w, int r0, int n) {
    extern __shared__ __align__(16) unsigned char zg_smem[];
    double2 (*Ls)[ZG_KC][ZG_T] = (double2 (*)[ZG_KC][ZG_T])zg_smem;                       // [stage][k][row]
    double2 (*Us)[ZG_KC][ZG_T] = (double2 (*)[ZG_KC][ZG_T])(zg_smem + 2 * ZG_KC * ZG_T * 16);  // [stage][k][col]
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int tr = r0 + blockIdx.x * ZG_T, tc = r0 + blockIdx.y * ZG_T;
    const int wr = (warp & 1) * 32, wc = (warp >> 1) * 16;  // warp tile: 32 complex rows x 16 cols
    double acc[8][2][2];
#pragma unroll
    for (int a = 0; a < 8; ++a)
#pragma unroll
        for (int b = 0; b < 2; ++b) acc[a][b][0] = acc[a][b][1] = 0.0;
    const int nchunks = (w + ZG_KC - 1) / ZG_KC;
    auto load = [&](int stage, int ch) {
        int kc = ch * ZG_KC;
        for (int idx = tid; idx < ZG_KC * ZG_T; idx += 256) {
            int r = idx % ZG_T, k = idx / ZG_T;
            int row = tr + r, kk = kc + k;
            bool ok = row < n && kk < w;
            cp_async16(&Ls[stage][k][r], A + (size_t)(k0 + (ok ? kk : 0)) * lda + (ok ? row : 0), ok);
        }
        for (int idx = tid; idx < ZG_KC * ZG_T; idx += 256) {
            int k = idx % ZG_KC, c = idx / ZG_KC;
            int col = tc + c, kk = kc + k;
            bool ok = col < n && kk < w;
            cp_async16(&Us[stage][k][c], A + (size_t)(ok ? col : 0) * lda + k0 + (ok ? kk : 0), ok);
        }
        cp_async_commit();
    };
    load(0, 0);
    for (int ch = 0; ch < nchunks; ++ch) {
        int st = ch & 1;
        if (ch + 1 < nchunks) {
            load(st ^ 1, ch + 1);
            cp_async_wait<1>();
        } else {
            cp_async_wait<0>();
        }
        __syncthreads();
#pragma unroll
        for (int ks = 0; ks < 2 * ZG_KC / 4; ++ks) {  // real k steps of 4
            int kr = ks * 4 + (lane & 3);
            int kc = kr >> 1, kp = kr & 1;
            double bfrag[2];
#pragma unroll
            for (int cb = 0; cb < 2; ++cb) {
                double2 u = Us[st][kc][wc + cb * 8 + (lane >> 2)];
                bfrag[cb] = kp ? u.y : u.x;
            }
#pragma unroll
            for (int rb = 0; rb < 8; ++rb) {
                int rr = rb * 8 + (lane >> 2);  // real row within the warp's 64
                int mu = wr + (rr >> 1), rp = rr & 1;
                double2 l = Ls[st][kc][mu];
                double a = (rp == kp) ? l.x : (rp == 0 ? -l.y : l.y);
#pragma unroll
                for (int cb = 0; cb < 2; ++cb) {
                    asm volatile(
                        "mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};"
                        : "+d"(acc[rb][cb][0]), "+d"(acc[rb][cb][1])
                        : "d"(a), "d"(bfrag[cb]));
                }
            }
        }
        __syncthreads();
    }
    // epilogue: lanes (l, l^4) hold the re/im rows of one complex row
    const bool even = ((lane >> 2) & 1) == 0;
    const int csel = 2 * (lane & 3) + (even ? 0 : 1);
    // two halves of 8 read-modify-writes, each with all its loads in flight before its stores
#pragma unroll
    for (int half = 0; half < 2; ++half) {
        double2 upd[4][2], old[4][2];
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            int rb = half * 4 + q;
#pragma unroll
            for (int cb = 0; cb < 2; ++cb) {
                double d0 = acc[rb][cb][0], d1 = acc[rb][cb][1];
                double p0 = __shfl_xor_sync(0xffffffffu, d0, 4), p1 = __shfl_xor_sync(0xffffffffu, d1, 4);
                upd[q][cb] = make_double2(even ? d0 : p1, even ? p0 : d1);
                int grow = tr + wr + ((rb * 8 + (lane >> 2)) >> 1), gcol = tc + wc + cb * 8 + csel;
                old[q][cb] = (grow < n && gcol < n) ? A[(size_t)gcol * lda + grow] : make_double2(0.0, 0.0);
            }
        }
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            int rb = half * 4 + q;
#pragma unroll
            for (int cb = 0; cb < 2; ++cb) {
                int grow = tr + wr + ((rb * 8 + (lane >> 2)) >> 1), gcol = tc + wc + cb * 8 + csel;
                if (grow < n && gcol < n)
                    A[(size_t)gcol * lda + grow] = make_double2(old[q][cb].x - upd[q][cb].x, old[q][cb].y - upd[q][cb].y);
            }
        }
    }
}

// ---- FP64 complex GEMM on DMMA, 128 x 64 complex tiles, 3-stage cp.async ring --------------
// The same real-embedding product as zgemm_dmma_kernel with a larger tile per CTA (8 warps in
// 4 x 2, warp tile 64 real rows x 32 columns: 32 m8n8k4 products per 4-deep real k step from
// 8 A and 4 B fragments; 64 accumulators per lane, ~200 registers, one CTA per SM) and K
// chunks of 8 complex in a 3-stage cp.async ring (24 KB per stage for 2 Mflop of products).
// A fragments come from the complex tile: the 32 lanes of a load touch 8
// distinct 16-byte entries (one shared-memory wavefront), and select Re, -Im or Im.
constexpr int ZH_M = 128;  // complex rows per CTA
constexpr int ZH_N = 64;   // columns per CTA
constexpr int ZH_KC = 8;   // complex K per stage
constexpr int ZH_STAGES = 3;
constexpr size_t ZH_SMEM = (size_t)ZH_STAGES * ZH_KC * (ZH_M + ZH_N) * sizeof(double2);

__global__ void __launch_bounds__(256, 1) zgemm_dmma_big_kernel(double2* A, size_t lda, int k0, int w, int r0, int n) {
    extern __shared__ __align__(16) unsigned char zh_smem[];
    double2 (*Ls)[ZH_KC][ZH_M] = (double2 (*)[ZH_KC][ZH_M])zh_smem;
    double2 (*Us)[ZH_KC][ZH_N] = (double2 (*)[ZH_KC][ZH_N])(zh_smem + (size_t)ZH_STAGES * ZH_KC * ZH_M * 16);
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int tr = r0 + blockIdx.x * ZH_M, tc = r0 + blockIdx.y * ZH_N;
    const int wr = (warp & 3) * 64, wc = (warp >> 2) * 32;  // real rows, columns of the warp tile
    double acc[8][4][2];
#pragma unroll
    for (int a = 0; a < 8; ++a)
#pragma unroll
        for (int b = 0; b < 4; ++b) acc[a][b][0] = acc[a][b][1] = 0.0;
    const int nchunks = (w + ZH_KC - 1) / ZH_KC;
    auto load = [&](int stage, int ch) {
        const int kc = ch * ZH_KC;
        for (int idx = tid; idx < ZH_KC * ZH_M; idx += 256) {
            const int r = idx % ZH_M, k = idx / ZH_M;
            const int row = tr + r, kk = kc + k;
            const bool ok = row < n && kk < w;
            cp_async16(&Ls[stage][k][r], A + (size_t)(k0 + (ok ? kk : 0)) * lda + (ok ? row : 0), ok);
        }
        for (int idx = tid; idx < ZH_KC * ZH_N; idx += 256) {
            const int k = idx % ZH_KC, c = idx / ZH_KC;
            const int col = tc + c, kk = kc + k;
            const bool ok = col < n && kk < w;
            cp_async16(&Us[stage][k][c], A + (size_t)(ok ? col : 0) * lda + k0 + (ok ? kk : 0), ok);
        }
    };
#pragma unroll
    for (int s = 0; s < ZH_STAGES - 1; ++s) {
        if (s < nchunks) load(s, s);
        cp_async_commit();
    }
    for (int ch = 0; ch < nchunks; ++ch) {
        const int st = ch % ZH_STAGES;
        if (ch + ZH_STAGES - 1 < nchunks) load((ch + ZH_STAGES - 1) % ZH_STAGES, ch + ZH_STAGES - 1);
        cp_async_commit();
        cp_async_wait<ZH_STAGES - 1>();
        __syncthreads();
#pragma unroll
        for (int ks = 0; ks < 2 * ZH_KC / 4; ++ks) {  // real k steps of 4
            const int kr = ks * 4 + (lane & 3);
            const int kc = kr >> 1, kp = kr & 1;
            double bfrag[4];
#pragma unroll
            for (int cb = 0; cb < 4; ++cb) {
                const double2 u = Us[st][kc][wc + cb * 8 + (lane >> 2)];
                bfrag[cb] = kp ? u.y : u.x;
            }
#pragma unroll
            for (int rb = 0; rb < 8; ++rb) {
                const int rr = wr + rb * 8 + (lane >> 2);
                const double2 l = Ls[st][kc][rr >> 1];
                const int rp = rr & 1;
                const double a = (rp == kp) ? l.x : (rp == 0 ? -l.y : l.y);
#pragma unroll
                for (int cb = 0; cb < 4; ++cb)
                    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};"
                                 : "+d"(acc[rb][cb][0]), "+d"(acc[rb][cb][1])
                                 : "d"(a), "d"(bfrag[cb]));
            }
        }
        __syncthreads();
    }
    cp_async_wait<0>();
    // epilogue: lanes (l, l ^ 4) hold the re/im rows of one complex row
    const bool even = ((lane >> 2) & 1) == 0;
    const int csel = 2 * (lane & 3) + (even ? 0 : 1);
#pragma unroll
    for (int rb = 0; rb < 8; ++rb) {
        double2 upd[4], old[4];
        const int grow = tr + ((wr + rb * 8 + (lane >> 2)) >> 1);
#pragma unroll
        for (int cb = 0; cb < 4; ++cb) {
            const double d0 = acc[rb][cb][0], d1 = acc[rb][cb][1];
            const double p0 = __shfl_xor_sync(0xffffffffu, d0, 4), p1 = __shfl_xor_sync(0xffffffffu, d1, 4);
            upd[cb] = make_double2(even ? d0 : p1, even ? p0 : d1);
            const int gcol = tc + wc + cb * 8 + csel;
            old[cb] = (grow < n && gcol < n) ? A[(size_t)gcol * lda + grow] : make_double2(0.0, 0.0);
        }
#pragma unroll
        for (int cb = 0; cb < 4; ++cb) {
            const int gcol = tc + wc + cb * 8 + csel;
            if (grow < n && gcol < n)
                A[(size_t)gcol * lda + grow] = make_double2(old[cb].x - upd[cb].x, old[cb].y - upd[cb].y);
        }
    }
}

// ---- FP32 complex GEMM on CUDA cores (fallback when tcgen05 is disabled) -----------------
__global__ void __launch_bounds__(256) cgemm_simt_kernel(float2* A, size_t lda, int k0, int w, int r0, int n) {
    __shared__ float2 Ls[ZG_KC][ZG_T + 1];
    __shared__ float2 Us[ZG_KC][ZG_T + 1];
    const int tid = threadIdx.x;
    const int tr = r0 + blockIdx.x * ZG_T, tc = r0 + blockIdx.y * ZG_T;
    const int ty = tid / 16, tx = tid % 16;  // 16 x 16 threads, 4 x 4 complex each
    float accr[4][4], acci[4][4];
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
        for (int b = 0; b < 4; ++b) accr[a][b] = acci[a][b] = 0.f;
    for (int kc = 0; kc < w; kc += ZG_KC) {
        for (int idx = tid; idx < ZG_KC * ZG_T; idx += 256) {
            int r = idx % ZG_T, k = idx / ZG_T;
            int row = tr + r, kk = kc + k;
            Ls[k][r] = (row < n && kk < w) ? A[(size_t)(k0 + kk) * lda + row] : make_float2(0.f, 0.f);
            int kq = idx % ZG_KC, c = idx / ZG_KC;
            int col = tc + c, kk2 = kc + kq;
            Us[kq][c] = (col < n && kk2 < w) ? A[(size_t)col * lda + k0 + kk2] : make_float2(0.f, 0.f);
        }
        __syncthreads();
#pragma unroll
        for (int k = 0; k < ZG_KC; ++k) {
            float2 lv[4], uv[4];
#pragma unroll
            for (int a = 0; a < 4; ++a) lv[a] = Ls[k][ty + 16 * a];
#pragma unroll
            for (int b = 0; b < 4; ++b) uv[b] = Us[k][tx + 16 * b];
#pragma unroll
            for (int a = 0; a < 4; ++a)
#pragma unroll
                for (int b = 0; b < 4; ++b) {
                    accr[a][b] = fmaf(lv[a].x, uv[b].x, fmaf(-lv[a].y, uv[b].y, accr[a][b]));
                    acci[a][b] = fmaf(lv[a].x, uv[b].y, fmaf(lv[a].y, uv[b].x, acci[a][b]));
                }
        }
        __syncthreads();
    }
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
        for (int b = 0; b < 4; ++b) {
            int row = tr + ty + 16 * a, col = tc + tx + 16 * b;
            if (row < n && col < n) {
                float2* c = A + (size_t)col * lda + row;
                float2 v = *c;
                v.x -= accr[a][b];
                v.y -= acci[a][b];
                *c = v;
            }
        }
}

// ---- host driver --------------------------------------------------------------------------
static int g_num_sms = 0;

template <typename R, int NB>
static size_t panel_smem(int chunk, int sub) {
    typedef typename Cx<R>::T C;
    return (size_t)chunk * (NB + 1) * sizeof(C) + (size_t)std::max(sub, 1) * NB * sizeof(C);
}

// The panel's grid barrier with one arrival missing: CTA 0 of a one-CTA grid waits for a
// second CTA that does not exist, gives up after limit_ns and records status 8, exactly as a
// factorization whose CTAs never meet would.
__global__ void barrier_selftest_kernel(unsigned* bar, int* status, unsigned long long limit_ns) {
    column_barrier(bar, 2u, status, limit_ns);
}

void launch_barrier_selftest(unsigned* bar, int* status, double limit_s, cudaStream_t st) {
    const double ns = std::min(std::max(limit_s, 0.0), 4.0) * 1e9;
    barrier_selftest_kernel<<<1, 32, 0, st>>>(bar, status, (unsigned long long)ns);
}

__global__ void perm_from_piv_kernel(const int* __restrict__ piv, int* __restrict__ perm, int n);

void lu_init_attributes() {
    static PerDeviceOnce done;
    once_per_device(done, [] {
        int dev;
        cudaGetDevice(&dev);
        int sms = 0;
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        g_num_sms = sms;
        cudaFuncSetAttribute(panel_kernel<double, 64, 0>, cudaFuncAttributeMaxDynamicSharedMemorySize, 220 * 1024);
        cudaFuncSetAttribute(panel_kernel<float, 128, 0>, cudaFuncAttributeMaxDynamicSharedMemorySize, 220 * 1024);
        cudaFuncSetAttribute(panel_kernel<double, 64, PANEL_SUB>, cudaFuncAttributeMaxDynamicSharedMemorySize, 220 * 1024);
        cudaFuncSetAttribute(panel_kernel<float, 128, PANEL_SUB>, cudaFuncAttributeMaxDynamicSharedMemorySize, 220 * 1024);
        cudaFuncSetAttribute(trsm_kernel<double, 64>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
        cudaFuncSetAttribute(trsm_kernel<float, 128>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
        cudaFuncSetAttribute(zgemm_dmma_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)ZG_SMEM);
        cudaFuncSetAttribute(zgemm_dmma_big_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)ZH_SMEM);
        cudaFuncSetAttribute(perm_from_piv_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
    });
}

size_t lu_workspace_bytes(int n, bool fp32) {
    (void)fp32;
    size_t P = 160;
    return (size_t)n * 2 * sizeof(int) + 64 + 2 * P * sizeof(Cand) + 2 * P * 128 * sizeof(double2) +
           2 * 128 * sizeof(double2) + 1024;
}

// Smallest slab of rows per panel CTA (TCU_PANEL_ROWS, default 32; the smem slab caps it).
static int panel_rows_per_cta() {
    static const int v = [] {
        const char* e = getenv("TCU_PANEL_ROWS");
        const int x = e ? atoi(e) : 0;
        return (x >= 16 && x <= 200) ? x : 32;
    }();
    return v;
}

// FP64 trailing update: 64 x 64 complex tiles, two CTAs per SM; TCU_FP64_GEMM=big selects the
// 128 x 64 tiles (one CTA per SM), measured 9% slower at 512 spheres (2211 vs 2029 ms of updates).
static bool fp64_big_tiles() {
    static const bool v = [] {
        const char* e = getenv("TCU_FP64_GEMM");
        return e && std::string(e) == "big";
    }();
    return v;
}

static bool panel_sub_enabled() {
    static const bool v = [] {
        const char* e = getenv("TCU_PANEL_SUB");
        return !(e && atoi(e) == 0);
    }();
    return v;
}

template <typename R, int NB>
static int run_panel(typename Cx<R>::T* A, int n, int k0, int w, LuWork& wk, cudaStream_t st) {
    typedef typename Cx<R>::T C;
    int rows = n - k0;
    // at least panel_rows_per_cta() rows per CTA: fewer CTAs arrive at each column's barrier
    const int per = wk.panel_rows > 0 ? wk.panel_rows : panel_rows_per_cta();
    int P = std::min(g_num_sms, std::max(1, (rows + per - 1) / per));
    int chunk = (rows + P - 1) / P;
    // 16-column sub-blocks when their pivot rows fit next to the slab (TCU_PANEL_SUB=0 turns
    // them off), else one rank-1 update per column over the whole panel
    int sub = panel_sub_enabled() ? PANEL_SUB : 0;
    if (sub && panel_smem<R, NB>(chunk, sub) > 220 * 1024) sub = 0;
    size_t smem = panel_smem<R, NB>(chunk, sub);
    if (smem > 220 * 1024) return 1;
    unsigned long long* keys = (unsigned long long*)wk.cand;  // 3 pivot words
    C* crow = (C*)(keys + 2 * 160);
    C* drow = crow + 2 * 160 * NB;
    cudaMemsetAsync(keys, 0, 4 * sizeof(unsigned long long), st);
    cudaMemsetAsync(wk.barrier, 0, 2 * sizeof(unsigned), st);
    size_t lda = (size_t)n;
    void* args[] = {&A, &lda, &k0, &n, &w, &chunk, &wk.piv, &wk.perm, &keys, &crow, &drow, &wk.barrier, &wk.status};
    void* fn = sub ? (void*)panel_kernel<R, NB, PANEL_SUB> : (void*)panel_kernel<R, NB, 0>;
    cudaError_t e = cudaLaunchCooperativeKernel(fn, dim3(P), dim3(PANEL_THREADS), args, smem, st);
    return e == cudaSuccess ? 0 : 2;
}

// perm from the interchanges: perm = iota, then swap perm[k] <-> perm[piv[k]] for k = 0..n-1
// in shared memory (one CTA; row i of P A is row perm[i] of A).
__global__ void perm_from_piv_kernel(const int* __restrict__ piv, int* __restrict__ perm, int n) {
    extern __shared__ int pm[];
    for (int i = threadIdx.x; i < n; i += blockDim.x) pm[i] = i;
    __syncthreads();
    if (threadIdx.x == 0)
        for (int k = 0; k < n; ++k) {
            int p = piv[k];
            if (p != k) {
                int t = pm[k];
                pm[k] = pm[p];
                pm[p] = t;
            }
        }
    __syncthreads();
    for (int i = threadIdx.x; i < n; i += blockDim.x) perm[i] = pm[i];
}

void launch_tf32_update(float2* A, int n, int k0, int w, LuWork& wk, cudaStream_t st, long long* launches);
void launch_tf32_update_region(float2* A, int n, int k0, int w, int r0, int m, int c0, int ncols, LuWork& wk,
                               cudaStream_t st, long long* launches);

// Mixed path: the trailing update of two consecutive 128-column panels in one K = 256 pass over
// A22 (TCU_LU_PAIRS=0: one update per panel). Panel a updates only panel b's columns; panel b,
// once factored, brings its own block rows up to date with panel a, and one update with both
// panels' L21 and U12 follows, so the trailing block is read and written once per 256 columns.
static bool lu_pairs_enabled() {
    static const bool v = [] {
        const char* e = getenv("TCU_LU_PAIRS");
        return !(e && atoi(e) == 0);
    }();
    return v;
}
bool launch_tf32_trsm_rhs(float2* A, int n, int k0, int w, LuWork& wk, cudaStream_t st, long long* launches);
void launch_tf32_trsm(float2* A, int n, int k0, int w, LuWork& wk, cudaStream_t st, long long* launches,
                      bool inverse_done, bool rhs_packed);
bool launch_tf32_trsm_inverse(float2* A, int n, int k0, int w, LuWork& wk, cudaStream_t st, cudaStream_t side,
                              long long* launches);

// A second stream of this thread and device (created once, kept for the process) on which the
// inverse of each step's L11 runs while the main stream applies the row interchanges: the
// inverse reads only the panel's diagonal block, the interchanges touch only the columns
// outside the panel.
struct SideStream {
    cudaStream_t stream = nullptr;
    cudaEvent_t panel_done = nullptr, inverse_done = nullptr;
    bool ok = false;
};
static SideStream* side_stream() {
    thread_local std::map<int, SideStream> by_device;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return nullptr;
    auto it = by_device.find(dev);
    if (it == by_device.end()) {
        SideStream s;
        s.ok = cudaStreamCreateWithFlags(&s.stream, cudaStreamNonBlocking) == cudaSuccess &&
               cudaEventCreateWithFlags(&s.panel_done, cudaEventDisableTiming) == cudaSuccess &&
               cudaEventCreateWithFlags(&s.inverse_done, cudaEventDisableTiming) == cudaSuccess;
        it = by_device.emplace(dev, s).first;
    }
    return it->second.ok ? &it->second : nullptr;
}

template <typename R, int NB>
static int lu_factor_impl(typename Cx<R>::T* A, int n, LuWork& wk, cudaStream_t st, long long* launches,
                          bool tensor_cores) {
    typedef typename Cx<R>::T C;
    lu_init_attributes();
    size_t lda = n;
    // (the FP16-piece packers hold one 128-column panel, so FP16 pieces keep one update per panel)
    const bool pairs = sizeof(R) == 4 && tensor_cores && !wk.f16_pieces && lu_pairs_enabled();
    int pend_k0 = -1, pend_w = 0;  // panel a whose update right of panel b is still pending
    for (int k0 = 0; k0 < n; k0 += NB) {
        int w = std::min(NB, n - k0);
        int rc;
        {
            StageScope sc(ST_PANEL, st);
            rc = run_panel<R, NB>(A, n, k0, w, wk, st);
        }
        ++*launches;
        if (rc) return rc;
        // the TRSM's inverse of L11 overlaps the row interchanges (mixed path)
        SideStream* side = (sizeof(R) == 4 && tensor_cores && k0 + w < n) ? side_stream() : nullptr;
        bool inverse_done = false;
        if (side && cudaEventRecord(side->panel_done, st) == cudaSuccess &&
            cudaStreamWaitEvent(side->stream, side->panel_done, 0) == cudaSuccess)
            inverse_done = launch_tf32_trsm_inverse((float2*)A, n, k0, w, wk, st, side->stream, launches) &&
                           cudaEventRecord(side->inverse_done, side->stream) == cudaSuccess;
        {
            StageScope sc(ST_SWAP, st);
            laswp_kernel<C><<<(n + 255) / 256, 256, 0, st>>>(A, lda, n, k0, w, wk.piv);
        }
        ++*launches;
        int r0 = k0 + w;
        int cols = n - r0;
        // work that does not need L11's inverse runs before the main stream waits for it: panel
        // b's block rows get panel a's update, then the TRSM's right-hand side is packed
        bool rhs_packed = false;
        if (sizeof(R) == 4 && tensor_cores && r0 < n) {
            if (pend_k0 >= 0)  // panel b: its block rows right of it get panel a's update first
                launch_tf32_update_region((float2*)A, n, pend_k0, pend_w, k0, w, r0, cols, wk, st, launches);
            rhs_packed = launch_tf32_trsm_rhs((float2*)A, n, k0, w, wk, st, launches);
        }
        if (inverse_done && cudaStreamWaitEvent(st, side->inverse_done, 0) != cudaSuccess) {
            cudaStreamSynchronize(side->stream);  // ordering by the host instead
        }
        if (r0 >= n) break;
        int cpc = 64;
        size_t smem = (size_t)NB * NB * sizeof(C);
        if (sizeof(R) == 4 && tensor_cores) {
            launch_tf32_trsm((float2*)A, n, k0, w, wk, st, launches, inverse_done, rhs_packed);
        } else {
            StageScope sc(ST_TRSM, st);
            trsm_kernel<R, NB><<<(cols + cpc - 1) / cpc, 256, smem, st>>>(A, lda, k0, w, n, cpc);
            ++*launches;
        }
        dim3 grid((cols + ZG_T - 1) / ZG_T, (cols + ZG_T - 1) / ZG_T);
        if constexpr (sizeof(R) == 8) {
            StageScope sc(ST_GEMM, st);
            if (fp64_big_tiles()) {
                dim3 g2((cols + ZH_M - 1) / ZH_M, (cols + ZH_N - 1) / ZH_N);
                zgemm_dmma_big_kernel<<<g2, 256, ZH_SMEM, st>>>((double2*)A, lda, k0, w, r0, n);
            } else {
                zgemm_dmma_kernel<<<grid, 256, ZG_SMEM, st>>>((double2*)A, lda, k0, w, r0, n);
            }
            ++*launches;
        } else {
            if (tensor_cores) {
                if (pend_k0 >= 0) {
                    // both panels' L21 and U12 (K = 256) over the trailing block at once
                    launch_tf32_update_region((float2*)A, n, pend_k0, pend_w + w, r0, cols, r0, cols, wk, st,
                                              launches);
                    pend_k0 = -1;
                } else if (pairs && cols > NB) {
                    // panel a: the next panel's columns now, the rest with panel b
                    launch_tf32_update_region((float2*)A, n, k0, w, r0, cols, r0, NB, wk, st, launches);
                    pend_k0 = k0;
                    pend_w = w;
                } else {
                    launch_tf32_update((float2*)A, n, k0, w, wk, st, launches);
                }
            } else {
                StageScope sc(ST_GEMM, st);
                cgemm_simt_kernel<<<grid, 256, 0, st>>>((float2*)A, lda, k0, w, r0, n);
                ++*launches;
            }
        }
    }
    {
        StageScope sc(ST_SWAP, st);
        perm_from_piv_kernel<<<1, 1024, (size_t)n * sizeof(int), st>>>(wk.piv, wk.perm, n);
        ++*launches;
    }
    return 0;
}

int lu_factor_fp64(double2* A, int n, LuWork& w, cudaStream_t st, long long* launches) {
    return lu_factor_impl<double, 64>(A, n, w, st, launches, false);
}
int lu_factor_fp32(float2* A, int n, LuWork& w, cudaStream_t st, long long* launches, bool tensor_cores) {
    return lu_factor_impl<float, 128>(A, n, w, st, launches, tensor_cores);
}

}  // namespace tcu
