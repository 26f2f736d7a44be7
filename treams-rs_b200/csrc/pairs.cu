// Sphere-pair kernels: Mie T blocks, incident plane waves, assembly of I - T C (FP64 or
// FP32 storage), the matrix-free operator (I - T C) x and the regular overlap O x used by
// the cross sections, and single translation blocks.
//
// Every pair (destination i, source j) needs the harmonic table
//   Z_ij[p*p+p+q] = z_p(k |r_i - r_j|) P_p^q(cos theta) e^{i q phi},  p <= 2 lmax,
// (sw/plan.rs:224-251) built by one warp: lane q computes order column q of the solid
// harmonics, multiplied by the radial sequence. Block entries are then the plan's term
// sums A = sum w Z[idx], B = sum w Z[idx] for each (source (l,m), destination (lambda,mu))
// and the helicity entries are A + B (pol 1) and A - B (pol 0) (sw/coupling.rs:127-140).
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>

#include "common.cuh"
#include "kernels.h"
#include "pairtable.cuh"
#include "plan.h"

namespace tcu {

template <typename OutT>
__device__ __forceinline__ void store_c(OutT* p, cplx v);
template <>
__device__ __forceinline__ void store_c<double2>(double2* p, cplx v) {
    __stcs(p, v);
}
template <>
__device__ __forceinline__ void store_c<float2>(float2* p, cplx v) {
    __stcs(p, make_float2(__double2float_rn(v.x), __double2float_rn(v.y)));
}

// ---- assembly of I - T C ----------------------------------------------------------------
// grid (N sources, ceil(N / pairs) destination groups), 256 threads. Thread item
// (destination i in the group, destination lm d) loops over source lm s and writes the
// four entries (2d..2d+1) x (2s..2s+1): coalesced 2-entry segments, contiguous over a warp.
// Out is column-major n x n with leading dimension ld; column j*M + e is source mode e of
// sphere j. T is N * L * 4 complex (mode-order 2x2 per degree, row-major).
// nsrc < nlm keeps only the first nsrc source lm of every sphere (the dipoles for nsrc = 3):
// the output then has 2 nsrc columns per source sphere.
template <typename OutT>
__global__ void __launch_bounds__(256) assemble_kernel(DevPlan P, int N, double k, const double* __restrict__ pos,
                                                       const cplx* __restrict__ T, OutT* __restrict__ out, size_t ld,
                                                       int pairs, int nsrc) {
    extern __shared__ cplx Zs[];  // pairs * tsize
    int j = blockIdx.x;
    int i0 = blockIdx.y * pairs;
    int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    int M = 2 * P.nlm;
    double xj = pos[3 * j], yj = pos[3 * j + 1], zj = pos[3 * j + 2];
    for (int w = warp; w < pairs; w += blockDim.x >> 5) {
        int i = i0 + w;
        if (i < N && i != j)
            pair_table(P, k, pos[3 * i] - xj, pos[3 * i + 1] - yj, pos[3 * i + 2] - zj, true, Zs + w * P.tsize, lane);
    }
    __syncthreads();
    int items = pairs * P.nlm;
    const int Mc = 2 * nsrc;
    for (int t = threadIdx.x; t < items; t += blockDim.x) {
        int il = t / P.nlm, d = t - il * P.nlm;
        int i = i0 + il;
        if (i >= N) continue;
        size_t row = (size_t)i * M + 2 * d;
        if (i == j) {
            for (int s = 0; s < nsrc; ++s) {
                size_t col = (size_t)j * Mc + 2 * s;
                cplx one = mk(s == d ? 1.0 : 0.0, 0.0), zero = mk(0.0, 0.0);
                store_c(out + col * ld + row, one);
                store_c(out + col * ld + row + 1, zero);
                store_c(out + (col + 1) * ld + row, zero);
                store_c(out + (col + 1) * ld + row + 1, one);
            }
            continue;
        }
        int lam = degree_of(d);
        const cplx* t4 = T + ((size_t)i * P.L + lam - 1) * 4;
        cplx t00 = t4[0], t01 = t4[1], t10 = t4[2], t11 = t4[3];
        const cplx* Z = Zs + il * P.tsize;
        for (int s = 0; s < nsrc; ++s) {
            cplx A, B;
            combo_sums(P, s * P.nlm + d, Z, A, B);
            cplx cp = cadd(A, B), cn = csub(A, B);
            size_t col = (size_t)j * Mc + 2 * s;
            store_c(out + col * ld + row, cneg(cmul(t00, cp)));
            store_c(out + col * ld + row + 1, cneg(cmul(t10, cp)));
            store_c(out + (col + 1) * ld + row, cneg(cmul(t01, cn)));
            store_c(out + (col + 1) * ld + row + 1, cneg(cmul(t11, cn)));
        }
    }
}

// ---- matrix-free operator ---------------------------------------------------------------
// y = zadd + alpha x + beta T (C x) (singular; T null: y = zadd + alpha x + beta C x) or
// y = x + R x (regular overlap, apply_t false, self block = identity). One CTA per destination sphere i; Q source
// spheres in flight, thread item (slot q, destination lm d) accumulates
// sum_s C[(d,pol),(s,pol)] x_j[(s,pol)] for p <= 8 columns; slots reduce in a fixed order.
constexpr int APPLY_MAXCOL = 8;
__global__ void __launch_bounds__(256) apply_kernel(DevPlan P, int N, double k, const double* __restrict__ pos,
                                                    const cplx* __restrict__ T, const cplx* __restrict__ x, size_t ldx,
                                                    int ncol, const cplx* __restrict__ zadd, double alpha, double beta,
                                                    bool singular, cplx* __restrict__ y, int Q) {
    extern __shared__ cplx smem[];
    cplx* Zs = smem;                                   // Q * tsize
    cplx* red = smem + (size_t)Q * P.tsize;            // Q * nlm * 2 * ncol (reduction)
    int i = blockIdx.x;
    int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    int M = 2 * P.nlm;
    int q = threadIdx.x / P.nlm, d = threadIdx.x - q * P.nlm;
    bool active = q < Q;
    cplx accp[APPLY_MAXCOL], accn[APPLY_MAXCOL];
    for (int c = 0; c < APPLY_MAXCOL; ++c) accp[c] = accn[c] = mk(0.0, 0.0);
    double xi = pos[3 * i], yi = pos[3 * i + 1], zi = pos[3 * i + 2];
    for (int j0 = 0; j0 < N; j0 += Q) {
        for (int w = warp; w < Q; w += blockDim.x >> 5) {
            int j = j0 + w;
            if (j < N && j != i)
                pair_table(P, k, xi - pos[3 * j], yi - pos[3 * j + 1], zi - pos[3 * j + 2], singular, Zs + w * P.tsize,
                           lane);
        }
        __syncthreads();
        int j = j0 + q;
        if (active && j < N && j != i) {
            const cplx* Z = Zs + q * P.tsize;
            for (int s = 0; s < P.nlm; ++s) {
                cplx A, B;
                combo_sums(P, s * P.nlm + d, Z, A, B);
                cplx cp = cadd(A, B), cn = csub(A, B);
                const cplx* xs = x + (size_t)j * M + 2 * s;
                for (int c = 0; c < ncol; ++c) {
                    cfma(accp[c], cp, xs[c * ldx]);
                    cfma(accn[c], cn, xs[c * ldx + 1]);
                }
            }
        }
        __syncthreads();
    }
    // fixed-order reduction over the Q slots
    if (active)
        for (int c = 0; c < ncol; ++c) {
            red[((size_t)q * P.nlm + d) * 2 * ncol + 2 * c] = accp[c];
            red[((size_t)q * P.nlm + d) * 2 * ncol + 2 * c + 1] = accn[c];
        }
    __syncthreads();
    for (int t = threadIdx.x; t < P.nlm * ncol; t += blockDim.x) {
        int dd = t % P.nlm, c = t / P.nlm;
        cplx sp = mk(0.0, 0.0), sn = mk(0.0, 0.0);
        for (int qq = 0; qq < Q; ++qq) {
            sp = cadd(sp, red[((size_t)qq * P.nlm + dd) * 2 * ncol + 2 * c]);
            sn = cadd(sn, red[((size_t)qq * P.nlm + dd) * 2 * ncol + 2 * c + 1]);
        }
        size_t row = (size_t)i * M + 2 * dd;
        cplx x0 = x[c * ldx + row], x1 = x[c * ldx + row + 1];
        cplx y0, y1;
        if (singular) {
            cplx tc0 = sp, tc1 = sn;  // T null: the coupling alone
            if (T) {
                int lam = degree_of(dd);
                const cplx* t4 = T + ((size_t)i * P.L + lam - 1) * 4;
                tc0 = cadd(cmul(t4[0], sp), cmul(t4[1], sn));
                tc1 = cadd(cmul(t4[2], sp), cmul(t4[3], sn));
            }
            y0 = cadd(cscale(x0, alpha), cscale(tc0, beta));
            y1 = cadd(cscale(x1, alpha), cscale(tc1, beta));
            if (zadd) {
                y0 = cadd(y0, zadd[c * ldx + row]);
                y1 = cadd(y1, zadd[c * ldx + row + 1]);
            }
        } else {
            y0 = cadd(x0, sp);
            y1 = cadd(x1, sn);
        }
        y[c * ldx + row] = y0;
        y[c * ldx + row + 1] = y1;
    }
}

// ---- matrix-free operator, slot-major mapping ----------------------------------------------
// Same sums as apply_kernel, with Q = 32 source slots per batch and thread t owning the slot
// q = t % 32 (its lane) and the destination modes d = t / 32 + 16 k: all lanes of a warp read
// the same plan term (one broadcast load, no divergence) against 32 different harmonic tables
// (table stride tsize = (2L+1)^2 entries, 4 banks apart mod 32: the minimum of 4 wavefronts per
// 16-byte load), and the batch's source coefficients are staged in shared memory with an odd
// row stride. Each thread sums its slot over all batches; slots are reduced in a fixed order.
constexpr int AP_Q = 32;
constexpr int AP_THREADS = 512;
template <int PASSES>  // ceil(nlm / 16) destination passes; at most 8 / PASSES columns
__global__ void __launch_bounds__(AP_THREADS) apply2_kernel(DevPlan P, int N, double k, const double* __restrict__ pos,
                                                     const cplx* __restrict__ T, const cplx* __restrict__ x,
                                                     size_t ldx, int ncol, const cplx* __restrict__ zadd, double alpha,
                                                     double beta, bool singular, cplx* __restrict__ y) {
    extern __shared__ cplx ap_smem[];
    const int nlm = P.nlm, M = 2 * nlm, XS = M + 1;  // odd row stride of the staged coefficients
    cplx* Zs = ap_smem;                              // AP_Q * tsize
    cplx* xs = Zs + (size_t)AP_Q * P.tsize;          // AP_Q * ncol * XS
    cplx* red = ap_smem;                             // at the end: AP_Q * nlm * 2 * ncol (aliases the above)
    const int i = blockIdx.x, tid = threadIdx.x;
    const int warp = tid >> 5, lane = tid & 31;
    const int q = tid % AP_Q, d0 = tid / AP_Q;       // d = d0 + 16 pass (16 warps)
    constexpr int COLS = APPLY_MAXCOL / PASSES;
    cplx accp[PASSES][COLS], accn[PASSES][COLS];
#pragma unroll
    for (int a = 0; a < PASSES; ++a)
#pragma unroll
        for (int c = 0; c < COLS; ++c) accp[a][c] = accn[a][c] = mk(0.0, 0.0);
    const double xi = pos[3 * i], yi = pos[3 * i + 1], zi = pos[3 * i + 2];
    for (int j0 = 0; j0 < N; j0 += AP_Q) {
        for (int w = warp; w < AP_Q; w += blockDim.x >> 5) {
            const int j = j0 + w;
            if (j < N && j != i)
                pair_table(P, k, xi - pos[3 * j], yi - pos[3 * j + 1], zi - pos[3 * j + 2], singular, Zs + w * P.tsize,
                           lane);
        }
        for (int t = tid; t < AP_Q * ncol * M; t += blockDim.x) {
            const int qq = t / (ncol * M), r = t - qq * ncol * M, c = r / M, e = r - c * M;
            const int j = j0 + qq;
            xs[((size_t)qq * ncol + c) * XS + e] = (j < N && j != i) ? x[c * ldx + (size_t)j * M + e] : mk(0.0, 0.0);
        }
        __syncthreads();
        const int j = j0 + q;
        if (j < N && j != i) {
            const cplx* Z = Zs + q * P.tsize;
            const cplx* xq = xs + (size_t)q * ncol * XS;
#pragma unroll
            for (int a = 0; a < PASSES; ++a) {
                const int d = d0 + 16 * a;
                if (d >= nlm) continue;
                for (int s = 0; s < nlm; ++s) {
                    cplx A, B;
                    combo_sums(P, s * nlm + d, Z, A, B);
                    const cplx cp = cadd(A, B), cn = csub(A, B);
#pragma unroll
                    for (int c = 0; c < COLS; ++c) {
                        if (c >= ncol) break;
                        cfma(accp[a][c], cp, xq[c * XS + 2 * s]);
                        cfma(accn[a][c], cn, xq[c * XS + 2 * s + 1]);
                    }
                }
            }
        }
        __syncthreads();
    }
    // fixed-order reduction over the slots
#pragma unroll
    for (int a = 0; a < PASSES; ++a) {
        const int d = d0 + 16 * a;
        if (d >= nlm) continue;
#pragma unroll
        for (int c = 0; c < COLS; ++c) {
            if (c >= ncol) break;
            red[((size_t)q * nlm + d) * 2 * ncol + 2 * c] = accp[a][c];
            red[((size_t)q * nlm + d) * 2 * ncol + 2 * c + 1] = accn[a][c];
        }
    }
    __syncthreads();
    for (int t = tid; t < nlm * ncol; t += blockDim.x) {
        const int dd = t % nlm, c = t / nlm;
        cplx sp = mk(0.0, 0.0), sn = mk(0.0, 0.0);
        for (int qq = 0; qq < AP_Q; ++qq) {
            sp = cadd(sp, red[((size_t)qq * nlm + dd) * 2 * ncol + 2 * c]);
            sn = cadd(sn, red[((size_t)qq * nlm + dd) * 2 * ncol + 2 * c + 1]);
        }
        const size_t row = (size_t)i * M + 2 * dd;
        const cplx x0 = x[c * ldx + row], x1 = x[c * ldx + row + 1];
        cplx y0, y1;
        if (singular) {
            cplx tc0 = sp, tc1 = sn;  // T null: the coupling alone
            if (T) {
                const int lam = degree_of(dd);
                const cplx* t4 = T + ((size_t)i * P.L + lam - 1) * 4;
                tc0 = cadd(cmul(t4[0], sp), cmul(t4[1], sn));
                tc1 = cadd(cmul(t4[2], sp), cmul(t4[3], sn));
            }
            y0 = cadd(cscale(x0, alpha), cscale(tc0, beta));
            y1 = cadd(cscale(x1, alpha), cscale(tc1, beta));
            if (zadd) {
                y0 = cadd(y0, zadd[c * ldx + row]);
                y1 = cadd(y1, zadd[c * ldx + row + 1]);
            }
        } else {
            y0 = cadd(x0, sp);
            y1 = cadd(x1, sn);
        }
        y[c * ldx + row] = y0;
        y[c * ldx + row + 1] = y1;
    }
}

// ---- expansion of a cluster into one global basis ----------------------------------------
// Regular translation blocks between every sphere and the origin o, cut from the blocks of
// the plan's lmax (the modes of a smaller lmax are a prefix of the mode order):
//   Ein  (n x Mg, ld n):   rows of sphere j = R(r_j <- o), local modes x global modes;
//   Eout (Mg x n, ld Mg):  columns of sphere i = R(o <- r_i), global modes x local modes.
// Entries between different helicities stay zero (the buffers are cleared first).
// grid (N, 2): y = 0 builds Ein, y = 1 Eout.
__global__ void __launch_bounds__(256) expand_kernel(DevPlan P, int N, double k, const double* __restrict__ pos,
                                                     double ox, double oy, double oz, int nlm_loc, int nlm_glob,
                                                     cplx* __restrict__ Ein, cplx* __restrict__ Eout) {
    extern __shared__ cplx ex_Z[];
    const int i = blockIdx.x, out_side = blockIdx.y;
    const double dx = pos[3 * i] - ox, dy = pos[3 * i + 1] - oy, dz = pos[3 * i + 2] - oz;
    if (threadIdx.x < 32) {
        if (out_side)
            pair_table(P, k, -dx, -dy, -dz, false, ex_Z, threadIdx.x);
        else
            pair_table(P, k, dx, dy, dz, false, ex_Z, threadIdx.x);
    }
    __syncthreads();
    const int Ml = 2 * nlm_loc, Mg = 2 * nlm_glob;
    const size_t n = (size_t)N * Ml;
    const int nd = out_side ? nlm_glob : nlm_loc, ns = out_side ? nlm_loc : nlm_glob;
    for (int t = threadIdx.x; t < nd * ns; t += blockDim.x) {
        const int s = t / nd, d = t - s * nd;
        cplx A, B;
        combo_sums(P, s * P.nlm + d, ex_Z, A, B);
        const cplx cp = cadd(A, B), cn = csub(A, B);
        if (out_side) {  // row 2d (+1) of the global modes, column i Ml + 2s (+1)
            cplx* c0 = Eout + ((size_t)i * Ml + 2 * s) * Mg;
            c0[2 * d] = cp;
            c0[Mg + 2 * d + 1] = cn;
        } else {  // row j Ml + 2d (+1), column 2s (+1) of the global modes
            cplx* c0 = Ein + (size_t)(2 * s) * n + (size_t)i * Ml;
            c0[2 * d] = cp;
            c0[n + 2 * d + 1] = cn;
        }
    }
}

// C (m x n) = A (m x k) B (k x n), complex FP64, column-major with leading dimensions; 16 x 16
// tiles through shared memory, fixed summation order.
__global__ void zgemm_small_kernel(int m, int n, int kk, const cplx* __restrict__ A, size_t lda,
                                   const cplx* __restrict__ B, size_t ldb, cplx* __restrict__ C, size_t ldc) {
    __shared__ cplx As[16][17], Bs[16][17];
    const int tx = threadIdx.x, ty = threadIdx.y;
    const int row = blockIdx.x * 16 + tx, col = blockIdx.y * 16 + ty;
    cplx acc = mk(0.0, 0.0);
    for (int k0 = 0; k0 < kk; k0 += 16) {
        As[ty][tx] = (row < m && k0 + ty < kk) ? A[(size_t)(k0 + ty) * lda + row] : mk(0.0, 0.0);
        Bs[ty][tx] = (col < n && k0 + tx < kk) ? B[(size_t)col * ldb + k0 + tx] : mk(0.0, 0.0);
        __syncthreads();
#pragma unroll
        for (int q = 0; q < 16; ++q) cfma(acc, As[q][tx], Bs[ty][q]);
        __syncthreads();
    }
    if (row < m && col < n) C[(size_t)col * ldc + row] = acc;
}

void launch_expand_blocks(const DevPlan& P, int N, double k, const double* pos, const double* origin, int nlm_loc,
                          int nlm_glob, cplx* Ein, cplx* Eout, cudaStream_t st) {
    expand_kernel<<<dim3(N, 2), 256, P.tsize * sizeof(cplx), st>>>(P, N, k, pos, origin[0], origin[1], origin[2],
                                                                  nlm_loc, nlm_glob, Ein, Eout);
}

void launch_zgemm_small(int m, int n, int k, const cplx* A, size_t lda, const cplx* B, size_t ldb, cplx* C,
                        size_t ldc, cudaStream_t st) {
    zgemm_small_kernel<<<dim3((m + 15) / 16, (n + 15) / 16), dim3(16, 16), 0, st>>>(m, n, k, A, lda, B, ldb, C, ldc);
}

// ---- single translation block (tests and the per-block API) -------------------------------
__global__ void block_kernel(DevPlan P, double k, double dx, double dy, double dz, bool singular, bool helicity,
                             cplx* out) {
    extern __shared__ cplx Z[];
    if (threadIdx.x < 32) pair_table(P, k, dx, dy, dz, singular, Z, threadIdx.x);
    __syncthreads();
    int M = 2 * P.nlm;
    for (int t = threadIdx.x; t < P.nlm * P.nlm; t += blockDim.x) {
        int s = t / P.nlm, d = t - s * P.nlm;
        cplx A, B;
        combo_sums(P, t, Z, A, B);
        // column-major M x M: entry (row to, col from) at col * M + row; pol 1 first
        size_t c1 = (size_t)(2 * s) * M, c0 = (size_t)(2 * s + 1) * M;
        int r1 = 2 * d, r0 = 2 * d + 1;
        if (helicity) {
            out[c1 + r1] = cadd(A, B);
            out[c1 + r0] = mk(0.0, 0.0);
            out[c0 + r1] = mk(0.0, 0.0);
            out[c0 + r0] = csub(A, B);
        } else {
            out[c1 + r1] = A;
            out[c0 + r0] = A;
            out[c1 + r0] = B;
            out[c0 + r1] = B;
        }
    }
}

// ---- Mie T blocks -----------------------------------------------------------------------
// Complex spherical Bessel j_l at complex z: power series below |z| = 0.5, else Miller's
// backward recurrence normalised by j_0 = sin z / z or j_1.
__device__ void cbessel_j_seq(int last, cplx z, cplx* out) {
    if (sqrt(cabs2(z)) < 0.5) {
        cplx sq = cmul(z, z), zl = mk(1.0, 0.0);
        double df = 1.0;
        for (int l = 0; l <= last; ++l) {
            if (l > 0) {
                zl = cmul(zl, z);
                df *= double(2 * l + 1);
            }
            cplx term = cscale(zl, 1.0 / df), sum = term;
            for (int q = 1; q < 24; ++q) {
                term = cscale(cmul(term, sq), -1.0 / (2.0 * q * (2.0 * (l + q) + 1.0)));
                sum = cadd(sum, term);
            }
            out[l] = sum;
        }
        return;
    }
    int start = last + 24 + int(2.0 * sqrt(cabs2(z)));
    cplx inv = cinv(z), fnext = mk(0.0, 0.0), f = mk(1e-200, 0.0);
    cplx keep[MAXP];
    for (int q = 0; q < MAXP; ++q) keep[q] = mk(0.0, 0.0);
    for (int kk = start; kk >= 1; --kk) {
        cplx fprev = csub(cscale(cmul(inv, f), double(2 * kk + 1)), fnext);
        fnext = f;
        f = fprev;
        if (cabs2(f) > 1e300) {
            f = cscale(f, 1e-150);
            fnext = cscale(fnext, 1e-150);
            for (int q = 0; q < MAXP; ++q) keep[q] = cscale(keep[q], 1e-150);
        }
        if (kk - 1 <= last) keep[kk - 1] = f;
        if (kk <= last) keep[kk] = fnext;
    }
    cplx s = csin(z), c = ccos(z);
    cplx j0 = cmul(s, inv), j1 = csub(cmul(cmul(s, inv), inv), cmul(c, inv));
    cplx scale = (cabs2(j0) >= cabs2(j1)) ? cdiv(j0, keep[0]) : cdiv(j1, keep[1]);
    for (int l = 0; l <= last; ++l) out[l] = cmul(keep[l], scale);
}

// One thread per (sphere, degree l): the 2x2 interface system of a homogeneous sphere
// (epsilon inside, vacuum outside) in helicity order, as in coeffs/mie.rs:133-251, then the
// swap into mode order (coeffs/mie.rs:123-130).
__global__ void mie_kernel(int L, double k0, int N, const double* __restrict__ radii, const cplx* __restrict__ eps,
                           cplx* __restrict__ T, int* __restrict__ status) {
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= N * L) return;
    int i = t / L, l = t % L + 1;
    double size = k0 * radii[i];
    cplx e = eps[i];
    cplx n_in = csqrt_p(e);
    cplx z_in = csqrt_p(cinv(e));  // sqrt(mu / eps), mu = 1
    cplx x_in = cscale(n_in, size);
    double x_out = size;
    // inner regular wave (f, f' + f/x) = (j_l, (l+1)/x j_l - j_{l+1})
    cplx jin[MAXP];
    cbessel_j_seq(l + 1, x_in, jin);
    cplx inv_in = cinv(x_in);
    cplx in0 = jin[l], in1 = csub(cscale(cmul(inv_in, jin[l]), double(l + 1)), jin[l + 1]);
    // outer regular and singular waves at real x_out
    double jo[MAXP];
    cplx ho[MAXP];
    bessel_j_sequence<MAXP>(l + 1, x_out, jo);
    hankel_sequence<MAXP>(l + 1, x_out, ho);
    double inv_out = 1.0 / x_out;
    cplx outw[2][2];  // [kind 0 regular, 1 singular][f, f' + f/x]
    outw[0][0] = mk(jo[l], 0.0);
    outw[0][1] = mk(double(l + 1) * inv_out * jo[l] - jo[l + 1], 0.0);
    outw[1][0] = ho[l];
    outw[1][1] = csub(cscale(ho[l], double(l + 1) * inv_out), ho[l + 1]);
    // impedance ratio z_out / z_in with z_out = 1
    cplx ratio = cinv(z_in);
    double sq = x_out * x_out;
    cplx q[4][2];
    for (int p = 0; p < 2; ++p)
        for (int qq = 0; qq < 2; ++qq) {
            double sign = (p == qq) ? 1.0 : -1.0;
            // a = (ratio + sign) / (2i) = -i (ratio + sign) / 2
            cplx rs = mk(ratio.x + sign, ratio.y);
            cplx a = mk(0.5 * rs.y, -0.5 * rs.x);
            cplx factor = cscale(a, sq);
            for (int ok = 0; ok < 2; ++ok) {
                const cplx* outer = outw[1 - ok];
                double os = (ok == 0) ? 1.0 : -1.0;
                cplx term = cscale(csub(cmul(outer[1], in0), cscale(cmul(outer[0], in1), sign)), os);
                q[p + ok * 2][qq] = cmul(term, factor);
            }
        }
    double scale = 0.0;
    for (int r = 0; r < 2; ++r)
        for (int c = 0; c < 2; ++c) scale = fmax(scale, fmax(fabs(q[r][c].x), fabs(q[r][c].y)));
    cplx a00 = cscale(q[0][0], 1.0 / scale), a01 = cscale(q[0][1], 1.0 / scale);
    cplx a10 = cscale(q[1][0], 1.0 / scale), a11 = cscale(q[1][1], 1.0 / scale);
    cplx det = csub(cmul(a00, a11), cmul(a01, a10));
    if (scale == 0.0 || !isfinite(scale) || cabs2(det) == 0.0) {
        atomicExch(status, 5);
        return;
    }
    cplx inv[2][2] = {{cscale(cdiv(a11, det), 1.0 / scale), cscale(cdiv(cneg(a01), det), 1.0 / scale)},
                      {cscale(cdiv(cneg(a10), det), 1.0 / scale), cscale(cdiv(a00, det), 1.0 / scale)}};
    cplx v[2][2];
    for (int r = 0; r < 2; ++r)
        for (int c = 0; c < 2; ++c) v[r][c] = cadd(cmul(q[2 + r][0], inv[0][c]), cmul(q[2 + r][1], inv[1][c]));
    cplx* o = T + ((size_t)i * L + l - 1) * 4;
    o[0] = v[1][1];
    o[1] = v[1][0];
    o[2] = v[0][1];
    o[3] = v[0][0];
    for (int r = 0; r < 4; ++r)
        if (!isfinite(o[r].x) || !isfinite(o[r].y)) atomicExch(status, 5);
}

// ---- incident plane waves ---------------------------------------------------------------
// Legendre factors F_l^m (sin^|m| factored out) by the recurrence of special/legendre.rs:26-59,
// angular factor tau + (2 pol - 1) pi, prefactor 2 sqrt(pi (2l+1)/(l(l+1))) sqrt((l-m)!/(l+m)!) i^l
// (pw/expand.rs:23-66), position phase e^{i k.r} (pw/field.rs:20-26).
__device__ cplx legendre_factor_pair(int l, int m, cplx z, cplx& lower) {
    int order = abs(m);
    lower = mk(0.0, 0.0);
    if (l < order) return mk(0.0, 0.0);
    cplx p = mk(1.0, 0.0);
    if (m >= 0)
        for (int q = 1; q <= m; ++q) p = cscale(p, -double(2 * q - 1));
    else
        for (int q = 1; q <= -m; ++q) p = cscale(p, 1.0 / double(2 * q));
    if (l == order) return p;
    cplx prev = p;
    p = cmul(p, cscale(z, double(2 * order + 1) / double(order - m + 1)));
    for (int q = order + 2; q <= l; ++q) {
        cplx next = cscale(csub(cscale(cmul(z, p), double(2 * q - 1)), cscale(prev, double(q + m - 1))), 1.0 / double(q - m));
        prev = p;
        p = next;
    }
    lower = prev;
    return p;
}
__device__ cplx cpowi(cplx z, int n) {
    if (n < 0) return cinv(cpowi(z, -n));
    cplx r = mk(1.0, 0.0);
    for (int q = 0; q < n; ++q) r = cmul(r, z);
    return r;
}

__global__ void plane_wave_kernel(int L, int N, const double* __restrict__ pos, int ncol, const cplx* __restrict__ kvecs,
                                  const int* __restrict__ pols, const double* __restrict__ lfac, cplx* __restrict__ out) {
    int M = 2 * L * (L + 2);
    size_t n = (size_t)N * M;
    size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n * ncol) return;
    int c = (int)(t / n);
    size_t row = t - (size_t)c * n;
    int i = (int)(row / M), e = (int)(row % M);
    int lm = e >> 1, mpol = (e & 1) ? 0 : 1;
    int l = degree_of(lm), m = lm + 1 - l * l - l;
    int pol = pols[c];
    if (mpol != pol) {
        out[t] = mk(0.0, 0.0);
        return;
    }
    cplx kx = kvecs[3 * c], ky = kvecs[3 * c + 1], kz = kvecs[3 * c + 2];
    cplx transverse = mk(0.0, 0.0), xy0 = mk(0.0, 0.0), xy1 = mk(0.0, 0.0);
    bool axis = (kx.x == 0.0 && kx.y == 0.0 && ky.x == 0.0 && ky.y == 0.0);
    if (!axis) {
        transverse = csqrt_p(cadd(cmul(kx, kx), cmul(ky, ky)));
        xy0 = cdiv(kx, transverse);
        xy1 = cdiv(ky, transverse);
    }
    cplx kk = csqrt_p(cadd(cadd(cmul(kx, kx), cmul(ky, ky)), cmul(kz, kz)));
    cplx azimuth = axis ? mk(1.0, 0.0) : cpowi(csub(xy0, mk(-xy1.y, xy1.x)), m);  // (xy0 - i xy1)^m
    cplx cosine = axis ? mk(cdiv(kz, kk).x >= 0.0 ? 1.0 : -1.0, 0.0) : cdiv(kz, kk);
    cplx sine = cdiv(transverse, kk);
    cplx pi = mk(0.0, 0.0), tau;
    if (m == 0) {
        cplx lower;
        tau = cmul(sine, legendre_factor_pair(l, 1, cosine, lower));
    } else {
        cplx lower, upper = legendre_factor_pair(l, m, cosine, lower);
        cplx power = cpowi(sine, abs(m) - 1);
        pi = cscale(cmul(power, upper), double(m));
        tau = cmul(power, csub(cscale(cmul(cosine, upper), double(l)), cscale(lower, double(l + m))));
    }
    cplx ang = cadd(tau, cscale(pi, 2.0 * pol - 1.0));
    // prefactor with i^l
    double norm = 2.0 * sqrt(M_PI * double(2 * l + 1) / double(l * (l + 1))) * lfac[l * l + l + m];
    cplx il;
    switch (l & 3) {
        case 0: il = mk(1, 0); break;
        case 1: il = mk(0, 1); break;
        case 2: il = mk(-1, 0); break;
        default: il = mk(0, -1); break;
    }
    cplx coef = cmul(cscale(il, norm), cmul(azimuth, ang));
    double ang_r = kx.x * pos[3 * i] + ky.x * pos[3 * i + 1] + kz.x * pos[3 * i + 2];
    double att = kx.y * pos[3 * i] + ky.y * pos[3 * i + 1] + kz.y * pos[3 * i + 2];
    double sc = exp(-att), sn, cs;
    sincos(ang_r, &sn, &cs);
    out[t] = cmul(coef, mk(sc * cs, sc * sn));
}

// ---- small vector kernels ---------------------------------------------------------------
// y = T x (block-diagonal 2x2 per (sphere, degree, order))
__global__ void apply_t_kernel(int L, int N, const cplx* __restrict__ T, const cplx* __restrict__ x, int ncol,
                               cplx* __restrict__ y) {
    int M = 2 * L * (L + 2);
    size_t n = (size_t)N * M;
    size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;  // one thread per row pair
    size_t pairs = n / 2;
    if (t >= pairs * ncol) return;
    int c = (int)(t / pairs);
    size_t rp = t - (size_t)c * pairs;
    size_t row = rp * 2;
    int i = (int)(row / M);
    int lm = (int)((row % M) >> 1);
    int l = degree_of(lm);
    const cplx* t4 = T + ((size_t)i * L + l - 1) * 4;
    cplx x0 = x[c * n + row], x1 = x[c * n + row + 1];
    y[c * n + row] = cadd(cmul(t4[0], x0), cmul(t4[1], x1));
    y[c * n + row + 1] = cadd(cmul(t4[2], x0), cmul(t4[3], x1));
}

// ---- host launchers ---------------------------------------------------------------------
int assemble_pairs_per_cta(int nlm) {
    int p = 256 / nlm;
    return p < 1 ? 1 : (p > 16 ? 16 : p);
}

void launch_assemble(const DevPlan& P, int N, double k, const double* pos, const cplx* T, void* out, size_t ld,
                     bool fp32, cudaStream_t st) {
    StageScope sc(ST_ASSEMBLE, st);
    int pairs = assemble_pairs_per_cta(P.nlm);
    dim3 grid(N, (N + pairs - 1) / pairs);
    size_t smem = (size_t)pairs * P.tsize * sizeof(cplx);
    if (fp32)
        assemble_kernel<float2><<<grid, 256, smem, st>>>(P, N, k, pos, T, (float2*)out, ld, pairs, P.nlm);
    else
        assemble_kernel<double2><<<grid, 256, smem, st>>>(P, N, k, pos, T, (double2*)out, ld, pairs, P.nlm);
}

static size_t apply2_smem(const DevPlan& P, int ncol) {
    const size_t main = ((size_t)AP_Q * P.tsize + (size_t)AP_Q * ncol * (2 * P.nlm + 1)) * sizeof(cplx);
    const size_t red = (size_t)AP_Q * P.nlm * 2 * ncol * sizeof(cplx);
    return std::max(main, red);
}

// Columns per launch of the slot-major kernel: its per-thread accumulators hold
// ceil(nlm / 16) destination passes x columns.
static int apply2_cols(const DevPlan& P) {
    int c = std::max(1, APPLY_MAXCOL / ((P.nlm + 15) / 16));
    while (c > 1 && apply2_smem(P, c) > 200 * 1024) --c;  // the shared-memory attribute
    return c;
}

void launch_apply(const DevPlan& P, int N, double k, const double* pos, const cplx* T, const cplx* x, size_t ldx,
                  int ncol, const cplx* zadd, double alpha, double beta, bool singular, cplx* y, cudaStream_t st) {
    StageScope sc(ST_APPLY, st);
    if (apply_gemm_supported(P)) {  // lmax 2..5: product form
        launch_apply_gemm(P, N, k, pos, T, x, ldx, ncol, zadd, alpha, beta, singular, y, st);
        return;
    }
    if (P.nlm > 64) {
        // lmax 8..10: the slot-major kernel's tables no longer fit; Q = 256 / nlm source slots
        // per CTA with one destination lm per thread
        const int Q = std::max(1, 256 / P.nlm);
        for (int c0 = 0; c0 < ncol; c0 += APPLY_MAXCOL) {
            const int nc = std::min(APPLY_MAXCOL, ncol - c0);
            const size_t smem = ((size_t)Q * P.tsize + (size_t)Q * P.nlm * 2 * nc) * sizeof(cplx);
            apply_kernel<<<N, 256, smem, st>>>(P, N, k, pos, T, x + (size_t)c0 * ldx, ldx, nc,
                                               zadd ? zadd + (size_t)c0 * ldx : nullptr, alpha, beta, singular,
                                               y + (size_t)c0 * ldx, Q);
        }
        return;
    }
    const int per = apply2_cols(P);
    for (int c0 = 0; c0 < ncol; c0 += per) {
        const int nc = std::min(per, ncol - c0);
        const cplx* xc = x + (size_t)c0 * ldx;
        const cplx* zc = zadd ? zadd + (size_t)c0 * ldx : nullptr;
        cplx* yc = y + (size_t)c0 * ldx;
        const size_t smem = apply2_smem(P, nc);
        switch ((P.nlm + 15) / 16) {
            case 1: apply2_kernel<1><<<N, AP_THREADS, smem, st>>>(P, N, k, pos, T, xc, ldx, nc, zc, alpha, beta, singular, yc); break;
            case 2: apply2_kernel<2><<<N, AP_THREADS, smem, st>>>(P, N, k, pos, T, xc, ldx, nc, zc, alpha, beta, singular, yc); break;
            case 3: apply2_kernel<3><<<N, AP_THREADS, smem, st>>>(P, N, k, pos, T, xc, ldx, nc, zc, alpha, beta, singular, yc); break;
            default: apply2_kernel<4><<<N, AP_THREADS, smem, st>>>(P, N, k, pos, T, xc, ldx, nc, zc, alpha, beta, singular, yc); break;
        }
    }
}

void launch_block(const DevPlan& P, double k, const double* d, bool singular, bool helicity, cplx* out,
                  cudaStream_t st) {
    block_kernel<<<1, 256, P.tsize * sizeof(cplx), st>>>(P, k, d[0], d[1], d[2], singular, helicity, out);
}

void launch_mie(int L, double k0, int N, const double* radii, const cplx* eps, cplx* T, int* status, cudaStream_t st) {
    StageScope sc(ST_MIE, st);
    int total = N * L;
    mie_kernel<<<(total + 127) / 128, 128, 0, st>>>(L, k0, N, radii, eps, T, status);
}

void launch_plane_wave(int L, int N, const double* pos, int ncol, const cplx* kvecs, const int* pols,
                       const double* lfac, cplx* out, cudaStream_t st) {
    size_t total = (size_t)N * 2 * L * (L + 2) * ncol;
    plane_wave_kernel<<<(unsigned)((total + 255) / 256), 256, 0, st>>>(L, N, pos, ncol, kvecs, pols, lfac, out);
}

void launch_apply_t(int L, int N, const cplx* T, const cplx* x, int ncol, cplx* y, cudaStream_t st) {
    size_t total = (size_t)N * L * (L + 2) * ncol;
    apply_t_kernel<<<(unsigned)((total + 255) / 256), 256, 0, st>>>(L, N, T, x, ncol, y);
}

void pairs_init_attributes() {
    cudaFuncSetAttribute(apply_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
    cudaFuncSetAttribute(apply2_kernel<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
    cudaFuncSetAttribute(apply2_kernel<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
    cudaFuncSetAttribute(apply2_kernel<3>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
    cudaFuncSetAttribute(apply2_kernel<4>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
    cudaFuncSetAttribute(assemble_kernel<double2>, cudaFuncAttributeMaxDynamicSharedMemorySize, 100 * 1024);
    cudaFuncSetAttribute(assemble_kernel<float2>, cudaFuncAttributeMaxDynamicSharedMemorySize, 100 * 1024);
    apply_gemm_init_attributes();
}

size_t apply_smem_bytes(const DevPlan& P, int ncol) { return apply2_smem(P, std::min(ncol, apply2_cols(P))); }

}  // namespace tcu
