// 2D Ewald lattice sums of outgoing spherical waves at an in-plane shift r (real wavenumber,
// real split) and the batched periodic-array solve X = (I - T S)^-1 T (one sphere per cell).
//
// D_lm(k, kpar, r) = sum'_R h_l(k|r+R|) Y_lm(-r-R) e^{i kpar.R} (lattice/mod.rs:11-15), with r
// first reduced into the cell (r' = r - R0, a factor e^{-i kpar.R0}; lattice/ewald.rs:610-665), is
// split at eta (lattice/ewald.rs:39-270) into
//   real space  sum_R e^{i kpar.R} Treal_lm(r'+R), Treal_lm(rho) = -i sqrt(2/pi) k^l |rho|^l
//               Y_lm(-rho/|rho|) I_2l(k|rho|, eta), R = 0 included for r' != 0 (real.rs:149-187)
//   reciprocal  sum_G pref_lm az^|m| sum_n (2 eta^2)^n/(sqrt2 eta) F_(1/2-n)(v, 0) S_lmn(beta^2)
//               with q = kpar + G, beta^2 = q.q/k^2, v = (beta^2 - 1)/(2 eta^2),
//               az = (q_x +- i q_y)/k, times e^{-i q.r'}             (lattice/reciprocal.rs:288-334)
//   self term   at l = 0, for r' = 0 only                            (lattice/reciprocal.rs:467-487)
// In the lattice plane only the n with s = 2n of S_lmn survive, so l - |m| odd sums vanish and
// n runs to (l - |m|)/2 (reciprocal.rs:22-60).
//
// Device layout: the real-space terms do not depend on the Bloch vector, so one launch
// tabulates Treal (NR x T complex, T = (lsum+1)^2) for the lattice points within the cutoff,
// and one CTA per Bloch vector then forms sum_R e^{i kpar.R} Treal_lm(R) (threads over lm,
// fixed order over R) plus the reciprocal sum over G in chunks of 256 points (threads over G
// evaluate F_n into shared memory, then threads over lm add the chunk in a fixed order).
// Results do not depend on the launch geometry or on timing.
//
// Special functions, all FP64 (each from a published method, checked against the binary128
// oracle to ~1e-14):
//   I_2l(z, eta) = eta^(2l+1)/2 sum_j c^j/j! R(l + 1/2 - j), c = 1/(2 eta^2), a = (z eta)^2/2,
//     R(d) = Gamma(d, a)/a^d (Kambe series, special/integrals/kambe.rs:36-120). R(d) for d >= 1/2
//     by the upward recurrence R(d+1) = (d R(d) + e^-a)/a from R(1/2) = sqrt(pi) erfc(sqrt a)/sqrt a
//     (all terms positive); for d < 1/2 by the power series (DLMF 8.7.3) where a < 2, else by
//     Legendre's continued fraction (DLMF 8.9.2, modified Lentz).
//   F_(1/2-n)(v, 0) = Gamma(1/2-n, v)/(-v)^(1/2-n) on the lower side of the cut
//     (lattice/reduced.rs:18-100): for v > 0, -i (-1)^n R(1/2-n, v); for v < 0 (propagating
//     orders, y = -v), Gamma(b)/y^b + i (-1)^n sum_k y^k/(k! (b+k)).
#include <cuda_runtime.h>

#include "common.cuh"
#include "kernels.h"
#include "smem_lu.cuh"

namespace tcu {

namespace {

constexpr int LS_JMAX = 64;                  // Kambe series terms
constexpr int LS_LADDER = LS_MAXL + 1 + LS_JMAX;
constexpr int LS_CHUNK = 256;                // reciprocal points per chunk

// Gamma(d, a)/a^d for real a > 0 and half-integer d < 1/2
__device__ double scaled_gamma_low(double d, double a) {
    if (a < 2.0) {
        // Gamma(d)/a^d - sum_k (-a)^k / (k! (d + k))
        double s = 1.0 / d, term = 1.0;
        for (int k = 1; k < 200; ++k) {
            term *= -a / k;
            double add = term / (d + k);
            s += add;
            if (k > a && fabs(add) < 1e-17 * fabs(s)) break;
        }
        return tgamma(d) * pow(a, -d) - s;
    }
    // e^-a / (a + 1 - d - 1(1-d)/(a + 3 - d - 2(2-d)/(a + 5 - d - ...)))
    const double tiny = 1e-300;
    double b = a + 1.0 - d, c = 1.0 / tiny, dd = 1.0 / b, h = dd;
    for (int i = 1; i < 400; ++i) {
        double an = -i * (i - d);
        b += 2.0;
        dd = an * dd + b;
        if (fabs(dd) < tiny) dd = tiny;
        c = b + an / c;
        if (fabs(c) < tiny) c = tiny;
        dd = 1.0 / dd;
        double del = dd * c;
        h *= del;
        if (fabs(del - 1.0) < 1e-16) break;
    }
    return exp(-a) * h;
}

// One warp per lattice point: Treal_lm(R) for every l <= lsum, |m| <= l.
__global__ void __launch_bounds__(128) real_table_kernel(int lsum, double k, double eta, int NR,
                                                         const double2* __restrict__ R, double sx, double sy,
                                                         const double* __restrict__ norm,
                                                         const double* __restrict__ reflection,
                                                         double2* __restrict__ tab) {
    __shared__ double ladder[4][LS_LADDER];
    __shared__ double kam[4][LS_MAXL + 1];
    __shared__ cplx Y[4][(LS_MAXL + 1) * (LS_MAXL + 1)];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int r = blockIdx.x * 4 + warp;
    if (r >= NR) return;
    const int T = (lsum + 1) * (lsum + 1);
    const double2 p = R[r];
    double dist, u[3];
    unit_direction(-p.x - sx, -p.y - sy, 0.0, dist, u);  // rho = -r' - R
    const double a = 0.5 * (k * dist * eta) * (k * dist * eta), c = 0.5 / (eta * eta);
    // ladder[i] = R(lsum + 1/2 - i)
    const int nlad = lsum + 1 + LS_JMAX;
    if (lane == 0) {
        double sa = sqrt(a), ea = exp(-a);
        double rr = 1.7724538509055160273 * erfc(sa) / sa;  // R(1/2)
        ladder[warp][lsum] = rr;
        double d = 0.5;
        for (int i = lsum - 1; i >= 0; --i) {
            rr = (d * rr + ea) / a;
            d += 1.0;
            ladder[warp][i] = rr;
        }
    }
    for (int i = lsum + 1 + lane; i < nlad; i += 32) ladder[warp][i] = scaled_gamma_low(lsum + 0.5 - i, a);
    if (lane <= lsum) solid_column(lsum, lane, u, reflection, Y[warp]);
    __syncwarp();
    if (lane <= lsum) {
        const int l = lane;
        double sum = 0.0, coef = 1.0;
        for (int j = 0; j < LS_JMAX; ++j) {
            if (j > 0) coef *= c / j;
            double term = coef * ladder[warp][lsum - l + j];
            sum += term;
            if (j > c + 3.0 && term <= 1e-17 * sum) break;
        }
        kam[warp][l] = 0.5 * pow(eta, 2 * l + 1) * sum;
    }
    __syncwarp();
    const double s2p = 0.79788456080286535588;  // sqrt(2/pi)
    for (int lm = lane; lm < T; lm += 32) {
        int l = (int)sqrt((double)lm);
        while (l * l > lm) --l;
        while ((l + 1) * (l + 1) <= lm) ++l;
        double f = s2p * pow(k * dist, (double)l) * norm[lm] * kam[warp][l];
        cplx y = Y[warp][lm];
        // -i f y
        tab[(size_t)r * T + lm] = mk(f * y.y, -f * y.x);
    }
}

// F'_n = (2 eta^2)^n / (sqrt 2 eta) F_(1/2-n)(v, 0), n = 0..nmax, real v != 0 (lower side)
__device__ void reduced_limits(int nmax, double v, double eta, cplx* out) {
    double factor = 1.0 / (1.4142135623730950488 * eta), step = 2.0 * eta * eta;
    if (v < 0.0) {
        double y = -v;
        for (int n = 0; n <= nmax; ++n) {
            double b = 0.5 - n;
            double s = 0.0, term = 1.0;
            for (int kk = 0; kk < 200; ++kk) {
                if (kk > 0) term *= y / kk;
                double add = term / (b + kk);
                s += add;
                if (kk > y && fabs(add) < 1e-18 * fabs(s)) break;
            }
            double re = tgamma(b) * pow(y, -b);
            double im = (n & 1) ? -s : s;
            out[n] = mk(factor * re, factor * im);
            factor *= step;
        }
    } else {
        for (int n = 0; n <= nmax; ++n) {
            double rr = scaled_gamma_low(0.5 - n, v);
            if (n == 0 && v >= 2.0) rr = 1.7724538509055160273 * erfc(sqrt(v)) / sqrt(v);
            // -i (-1)^n R
            double im = (n & 1) ? rr : -rr;
            out[n] = mk(0.0, factor * im);
            factor *= step;
        }
    }
}

// One CTA per Bloch vector. smem: phases NR double2, chunk arrays.
__global__ void __launch_bounds__(256) lattice_sum_kernel(LatticeSumArgs A) {
    extern __shared__ double2 ls_smem[];
    double2* ph = ls_smem;                               // NR
    double2* gF = ph + A.NR;                             // LS_CHUNK * (nmax + 1)
    double2* gaz = gF + LS_CHUNK * (A.lsum / 2 + 1);     // LS_CHUNK
    double2* gph = gaz + LS_CHUNK;                       // LS_CHUNK: e^{-i q.r'}
    double* gb2 = (double*)(gph + LS_CHUNK);             // LS_CHUNK
    const int T = (A.lsum + 1) * (A.lsum + 1), nmax = A.lsum / 2;
    const int tid = threadIdx.x;
    for (int kp = blockIdx.x; kp < A.nk; kp += gridDim.x) {
        const double2 kpar = A.kpar[kp];
        for (int r = tid; r < A.NR; r += blockDim.x) {
            double2 R = A.R[r];
            double s, c;
            sincos(kpar.x * R.x + kpar.y * R.y, &s, &c);
            ph[r] = mk(c, s);
        }
        __syncthreads();
        int lm = tid, l = 0, m = 0;
        bool active = lm < T;
        if (active) {
            while ((l + 1) * (l + 1) <= lm) ++l;
            m = lm - l * l - l;
        }
        const int am = m < 0 ? -m : m;
        const bool even = ((l - am) & 1) == 0;
        cplx acc = mk(0.0, 0.0);
        if (active)
            for (int r = 0; r < A.NR; ++r) cfma(acc, __ldg(&A.realtab[(size_t)r * T + lm]), ph[r]);
        cplx rec = mk(0.0, 0.0);
        for (int g0 = 0; g0 < A.NG; g0 += LS_CHUNK) {
            __syncthreads();
            int g = g0 + tid;
            if (tid < LS_CHUNK && g < A.NG) {
                double2 G = A.G[g];
                double qx = kpar.x + G.x, qy = kpar.y + G.y;
                double b2 = (qx * qx + qy * qy) / (A.k * A.k);
                double v = (b2 - 1.0) / (2.0 * A.eta * A.eta);
                if (fabs(v) <= 1e-14) {
                    atomicExch(A.status, 9);  // on a diffraction threshold (reciprocal.rs:236-241)
                    for (int n = 0; n <= nmax; ++n) gF[tid * (nmax + 1) + n] = mk(0.0, 0.0);
                } else {
                    reduced_limits(nmax, v, A.eta, gF + tid * (nmax + 1));
                }
                gb2[tid] = b2;
                gaz[tid] = mk(qx / A.k, qy / A.k);
                double ps, pc;
                sincos(-(qx * A.sx + qy * A.sy), &ps, &pc);
                gph[tid] = mk(pc, ps);
            }
            __syncthreads();
            if (active && even) {
                const int nm = (l - am) / 2;
                const double* coef = A.coef + (size_t)lm * LS_NMAX;
                const int cnt = min(LS_CHUNK, A.NG - g0);
                for (int t = 0; t < cnt; ++t) {
                    const double b2 = gb2[t];
                    const double2* F = gF + t * (nmax + 1);
                    cplx s = mk(0.0, 0.0);
                    for (int n = 0; n <= nm; ++n) {  // Horner in beta^2
                        s = cscale(s, b2);
                        cfma(s, mk(coef[n], 0.0), F[n]);
                    }
                    cplx az = gaz[t];
                    if (m < 0) az.y = -az.y;
                    cplx azm = mk(1.0, 0.0);
                    for (int q = 0; q < am; ++q) azm = cmul(azm, az);
                    cfma(rec, s, cmul(azm, gph[t]));
                }
            }
        }
        if (active) {
            cplx v = cadd(acc, cmul(A.pref[lm], rec));
            if (lm == 0) v = cadd(v, A.self0);
            double cs, cc;  // e^{-i kpar.R0} of the shift reduced into the cell
            sincos(-(kpar.x * A.R0x + kpar.y * A.R0y), &cs, &cc);
            A.out[(size_t)kp * A.ldo + lm] = cmul(v, mk(cc, cs));
        }
        __syncthreads();
    }
}

// ---- blocked shared-memory LU of the periodic-array kernel -------------------------------
// A (M x M column-major, shared, M <= 128) = P^T L U with partial pivoting (largest modulus,
// lowest row on ties), in panels of BP = 16 columns: warp 0 factors the panel (pivot search by
// shuffles, swaps, scaling and rank-1 updates inside the panel with warp-level synchronisation
// only), then every thread applies the panel's interchanges to the other columns, forms
// U12 = L11^-1 A12 (thread per column) and the rank-16 trailing update (4 x 2 register tiles).
// dinv receives 1 / U[i][i]. Returns false on every thread for an exactly zero pivot.
constexpr int BP = 16;

// X[j][i] -= sum_{c in [k0, k1)} A[c][i] X[j][c] for rows i in [r0, r1) and columns j in
// [j0, j1) (column-major, leading dimension M). Each thread owns a 4-row x 2-column register
// tile, so a step over c loads 6 entries for 8 products (the shared-memory traffic, not the
// arithmetic, bounds these updates).
__device__ void tile_update(const double2* A, double2* X, int M, int r0, int r1, int j0, int j1, int k0, int k1) {
    const int rows = r1 - r0, cols = j1 - j0;
    if (rows <= 0 || cols <= 0) return;
    const int tr = (rows + 3) / 4, tc = (cols + 1) / 2;
    for (int t = threadIdx.x; t < tr * tc; t += blockDim.x) {
        const int i0 = r0 + 4 * (t % tr), jj = j0 + 2 * (t / tr);
        cplx acc[4][2];
#pragma unroll
        for (int a = 0; a < 4; ++a) acc[a][0] = acc[a][1] = mk(0.0, 0.0);
        for (int c = k0; c < k1; ++c) {
            cplx l[4], u[2];
#pragma unroll
            for (int a = 0; a < 4; ++a) l[a] = i0 + a < r1 ? A[c * M + i0 + a] : mk(0.0, 0.0);
#pragma unroll
            for (int b = 0; b < 2; ++b) u[b] = jj + b < j1 ? X[(jj + b) * M + c] : mk(0.0, 0.0);
#pragma unroll
            for (int a = 0; a < 4; ++a)
#pragma unroll
                for (int b = 0; b < 2; ++b) cfma(acc[a][b], l[a], u[b]);
        }
#pragma unroll
        for (int a = 0; a < 4; ++a)
#pragma unroll
            for (int b = 0; b < 2; ++b)
                if (i0 + a < r1 && jj + b < j1) X[(jj + b) * M + i0 + a] = csub(X[(jj + b) * M + i0 + a], acc[a][b]);
    }
}

__device__ bool blocked_lu(double2* A, int M, int* piv, double2* dinv, int* sing) {
    const int tid = threadIdx.x, nth = blockDim.x, lane = tid & 31, warp = tid >> 5;
    if (tid == 0) *sing = 0;
    __syncthreads();
    for (int k0 = 0; k0 < M; k0 += BP) {
        const int w = min(BP, M - k0), k1 = k0 + w;
        if (warp == 0) {
            for (int c = k0; c < k1; ++c) {
                double best = -1.0;
                int bi = c;
                for (int i = c + lane; i < M; i += 32) {
                    const double v = cabs2(A[c * M + i]);
                    if (v > best) {
                        best = v;
                        bi = i;
                    }
                }
                for (int off = 16; off > 0; off >>= 1) {
                    const double ov = __shfl_xor_sync(0xffffffffu, best, off);
                    const int oi = __shfl_xor_sync(0xffffffffu, bi, off);
                    if (ov > best || (ov == best && oi < bi)) {
                        best = ov;
                        bi = oi;
                    }
                }
                if (lane == 0) {
                    piv[c] = bi;
                    if (!(best > 0.0)) *sing = 1;
                }
                if (bi != c && lane < w) {  // swap rows c and bi inside the panel
                    const int j = k0 + lane;
                    const double2 t = A[j * M + c];
                    A[j * M + c] = A[j * M + bi];
                    A[j * M + bi] = t;
                }
                __syncwarp();
                const cplx d = A[c * M + c];
                if (cabs2(d) > 0.0) {
                    const cplx inv = cinv(d);
                    if (lane == 0) dinv[c] = inv;
                    for (int i = c + 1 + lane; i < M; i += 32) A[c * M + i] = cmul(A[c * M + i], inv);
                    __syncwarp();
                    for (int j = c + 1; j < k1; ++j) {
                        const cplx u = cneg(A[j * M + c]);
                        for (int i = c + 1 + lane; i < M; i += 32) {
                            cplx v = A[j * M + i];
                            cfma(v, A[c * M + i], u);
                            A[j * M + i] = v;
                        }
                    }
                }
                __syncwarp();
            }
        }
        __syncthreads();
        if (*sing) return false;
        // interchanges of the panel on the columns outside it, in pivot order
        for (int j = tid; j < M; j += nth) {
            if (j >= k0 && j < k1) continue;
            for (int c = k0; c < k1; ++c) {
                const int pr = piv[c];
                if (pr != c) {
                    const double2 t = A[j * M + c];
                    A[j * M + c] = A[j * M + pr];
                    A[j * M + pr] = t;
                }
            }
        }
        __syncthreads();
        // U12 = L11^-1 A12, one thread per column
        for (int j = k1 + tid; j < M; j += nth)
            for (int r = k0 + 1; r < k1; ++r) {
                cplx v = A[j * M + r];
                for (int c = k0; c < r; ++c) cfma(v, cneg(A[c * M + r]), A[j * M + c]);
                A[j * M + r] = v;
            }
        __syncthreads();
        // A22 -= L21 U12
        tile_update(A, A, M, k1, M, k1, M, k0, k1);
        __syncthreads();
    }
    return true;
}

// B (M x nc, shared) <- U^-1 L^-1 P B with the factors of blocked_lu: the interchanges (thread
// per column), then blocks of BP rows: the block's triangle (thread per column) and the update
// of the remaining rows (4 x 2 register tiles), forward with L and backward with U.
__device__ void blocked_lu_solve(const double2* A, int M, const int* piv, const double2* dinv, double2* B, int nc) {
    const int tid = threadIdx.x, nth = blockDim.x;
    for (int j = tid; j < nc; j += nth)
        for (int c = 0; c < M; ++c) {
            const int pr = piv[c];
            if (pr != c) {
                const double2 t = B[j * M + c];
                B[j * M + c] = B[j * M + pr];
                B[j * M + pr] = t;
            }
        }
    __syncthreads();
    for (int k0 = 0; k0 < M; k0 += BP) {  // L y = b
        const int k1 = min(M, k0 + BP);
        for (int j = tid; j < nc; j += nth)
            for (int r = k0 + 1; r < k1; ++r) {
                cplx v = B[j * M + r];
                for (int c = k0; c < r; ++c) cfma(v, cneg(A[c * M + r]), B[j * M + c]);
                B[j * M + r] = v;
            }
        __syncthreads();
        tile_update(A, B, M, k1, M, 0, nc, k0, k1);
        __syncthreads();
    }
    for (int k1 = M; k1 > 0; k1 -= BP) {  // U x = y
        const int k0 = max(0, k1 - BP);
        for (int j = tid; j < nc; j += nth)
            for (int r = k1 - 1; r >= k0; --r) {
                cplx v = B[j * M + r];
                for (int c = r + 1; c < k1; ++c) cfma(v, cneg(A[c * M + r]), B[j * M + c]);
                B[j * M + r] = cmul(v, dinv[r]);
            }
        __syncthreads();
        tile_update(A, B, M, 0, k0, 0, nc, k0, k1);
        __syncthreads();
    }
}

// ---- batched periodic-array solve ----------------------------------------------------------
// One CTA per Bloch vector: Z = D/N (harmonic table), A = I - T S in shared memory (S from the
// translation plan, cluster/interaction.rs:292-315 with sw/plan.rs:383-413 evaluate_periodic),
// blocked partial-pivot LU in shared memory, then X = A^-1 T in panels of 48 right-hand sides.
constexpr int AS_PANEL = 48;

__global__ void __launch_bounds__(512) array_solve_kernel(DevPlan P, const double2* __restrict__ D, size_t ldd,
                                                          const double* __restrict__ norm,
                                                          const double2* __restrict__ Tm, int nk,
                                                          double2* __restrict__ X, int* __restrict__ status) {
    extern __shared__ double2 as_smem[];
    const int M = 2 * P.nlm;
    double2* A = as_smem;                  // M x M column-major
    double2* B = A + M * M;                // M x AS_PANEL column-major; the harmonic table aliases it
    __shared__ int piv[128];
    __shared__ double2 dinv[128];
    __shared__ int sing;
    const int tid = threadIdx.x, nth = blockDim.x;
    for (int kp = blockIdx.x; kp < nk; kp += gridDim.x) {
        double2* Z = B;
        for (int t = tid; t < P.tsize; t += nth) {
            double2 d = D[(size_t)kp * ldd + t];
            Z[t] = cscale(d, 1.0 / norm[t]);
        }
        __syncthreads();
        // A = I - T S: item (s, d) writes rows 2d, 2d+1 of columns 2s, 2s+1
        for (int it = tid; it < P.nlm * P.nlm; it += nth) {
            int s = it / P.nlm, d = it - s * P.nlm;
            int lam = 1;
            while ((lam + 1) * (lam + 1) - 1 <= d) ++lam;
            const double2* t4 = Tm + (lam - 1) * 4;
            cplx Aa, Bb;
            plan_combo_sums(P, s * P.nlm + d, Z, Aa, Bb);
            cplx cp = cadd(Aa, Bb), cn = csub(Aa, Bb);
            double one = s == d ? 1.0 : 0.0;
            cplx a00 = cmul(t4[0], cp), a10 = cmul(t4[2], cp), a01 = cmul(t4[1], cn), a11 = cmul(t4[3], cn);
            A[(2 * s) * M + 2 * d] = mk(one - a00.x, -a00.y);
            A[(2 * s) * M + 2 * d + 1] = cneg(a10);
            A[(2 * s + 1) * M + 2 * d] = cneg(a01);
            A[(2 * s + 1) * M + 2 * d + 1] = mk(one - a11.x, -a11.y);
        }
        __syncthreads();
        if (!blocked_lu(A, M, piv, dinv, &sing)) {
            if (tid == 0) atomicExch(status, 5);
            __syncthreads();
            continue;
        }
        // X = U^-1 L^-1 P T, panels of AS_PANEL columns
        double2* Xk = X + (size_t)kp * M * M;
        for (int c0 = 0; c0 < M; c0 += AS_PANEL) {
            const int nc = min(AS_PANEL, M - c0);
            // B = T (block diagonal: columns 2i, 2i+1 of mode pair i carry t[.][0], t[.][1])
            for (int it = tid; it < M * nc; it += nth) {
                int jj = it / M, i = it - jj * M, col = c0 + jj;
                cplx v = mk(0.0, 0.0);
                if ((i >> 1) == (col >> 1)) {
                    int lm = col >> 1, lam = 1;
                    while ((lam + 1) * (lam + 1) - 1 <= lm) ++lam;
                    v = Tm[(lam - 1) * 4 + (i & 1) * 2 + (col & 1)];
                }
                B[jj * M + i] = v;
            }
            __syncthreads();
            blocked_lu_solve(A, M, piv, dinv, B, nc);
            for (int it = tid; it < M * nc; it += nth) {
                int jj = it / M, i = it - jj * M;
                Xk[(size_t)(c0 + jj) * M + i] = B[jj * M + i];
            }
            __syncthreads();
        }
    }
}

}  // namespace

void launch_real_table(int lsum, double k, double eta, int NR, const double2* R, double sx, double sy,
                       const double* norm, const double* reflection, double2* tab, cudaStream_t st) {
    StageScope sc(ST_LATTICE, st);
    real_table_kernel<<<(NR + 3) / 4, 128, 0, st>>>(lsum, k, eta, NR, R, sx, sy, norm, reflection, tab);
}

size_t lattice_sum_smem(int lsum, int NR) {
    return (size_t)NR * 16 + (size_t)LS_CHUNK * (lsum / 2 + 1) * 16 + 2 * LS_CHUNK * 16 + LS_CHUNK * 8;
}

void launch_lattice_sum(const LatticeSumArgs& a, int grid, cudaStream_t st) {
    StageScope sc(ST_LATTICE, st);
    size_t smem = lattice_sum_smem(a.lsum, a.NR);
    cudaFuncSetAttribute(lattice_sum_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    lattice_sum_kernel<<<grid, 256, smem, st>>>(a);
}

size_t array_solve_smem(int L) {
    int M = 2 * L * (L + 2);
    return (size_t)M * M * 16 + (size_t)M * AS_PANEL * 16;
}

void launch_array_solve(const DevPlan& P, const double2* D, size_t ldd, const double* norm, const double2* Tm, int nk,
                        double2* X, int* status, int grid, cudaStream_t st) {
    StageScope sc(ST_SMALL_LU, st);
    size_t smem = array_solve_smem(P.L);
    cudaFuncSetAttribute(array_solve_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    array_solve_kernel<<<grid, 512, smem, st>>>(P, D, ldd, norm, Tm, nk, X, status);
}

}  // namespace tcu
