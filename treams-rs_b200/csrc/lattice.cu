// 2D Ewald lattice sums of outgoing spherical waves at a shift r (real wavenumber, real split)
// and the batched periodic-array solve X = (I - T S)^-1 T (one sphere per cell).
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
// n runs to (l - |m|)/2 (reciprocal.rs:22-60). Off the plane (r_z != 0) n runs to l - |m|,
// S_lmn = sum_s (-k r_z)^(2n-s) beta^(l-|m|-s) / ((2n-s)! (s-n)! ((l+|m|-s)/2)! ((l-|m|-s)/2)!)
// over n <= s <= min(l - |m|, 2n) with l - |m| - s even, and F_(1/2-n)(v, 0) becomes
// F_(1/2-n)(v, t) = sum_j (t/2)^j / j! F_(1/2-n-j)(v, 0), t = (k r_z eta)^2 (reduced.rs:223).
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
                                                         double sz, const double* __restrict__ norm,
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
    unit_direction(-p.x - sx, -p.y - sy, -sz, dist, u);  // rho = -r' - R
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

// F_(1/2-n)(v, 0) on the lower side of the cut, real v != 0 (the terms of reduced_limits
// without the factor (2 eta^2)^n / (sqrt 2 eta))
__device__ cplx reduced_limit(int n, double v) {
    if (v < 0.0) {
        const double y = -v, b = 0.5 - n;
        double s = 0.0, term = 1.0;
        for (int kk = 0; kk < 200; ++kk) {
            if (kk > 0) term *= y / kk;
            double add = term / (b + kk);
            s += add;
            if (kk > y && fabs(add) < 1e-18 * fabs(s)) break;
        }
        return mk(tgamma(b) * pow(y, -b), (n & 1) ? -s : s);
    }
    double rr = scaled_gamma_low(0.5 - n, v);
    if (n == 0 && v >= 2.0) rr = 1.7724538509055160273 * erfc(sqrt(v)) / sqrt(v);
    return mk(0.0, (n & 1) ? rr : -rr);  // -i (-1)^n R
}

// Off the lattice plane (lattice/reduced.rs:223): F'_n = (2 eta^2)^n / (sqrt 2 eta) F_(1/2-n)(v, t)
// with F_(1/2-n)(v, t) = sum_j (t/2)^j / j! F_(1/2-n-j)(v, 0), j = 0..J (tw[j] = (t/2)^j / j!),
// n = 0..nmax. Each limit is evaluated once and added to every n it reaches, in increasing j.
__device__ void reduced_shifted(int nmax, int J, const double* tw, double v, double eta, cplx* out) {
    for (int n = 0; n <= nmax; ++n) out[n] = mk(0.0, 0.0);
    for (int i = 0; i <= nmax + J; ++i) {
        const cplx L = reduced_limit(i, v);
        for (int n = min(nmax, i); n >= max(0, i - J); --n) cfma(out[n], mk(tw[i - n], 0.0), L);
    }
    double factor = 1.0 / (1.4142135623730950488 * eta);
    const double step = 2.0 * eta * eta;
    for (int n = 0; n <= nmax; ++n) {
        out[n] = cscale(out[n], factor);
        factor *= step;
    }
}

// One CTA per Bloch vector. smem: phases NR double2, chunk arrays.
__global__ void __launch_bounds__(256) lattice_sum_kernel(LatticeSumArgs A) {
    extern __shared__ double2 ls_smem[];
    __shared__ double tw[LS_TMAX + 1];                   // (t/2)^j / j! off the plane
    const int nF = A.offplane ? A.lsum + 1 : A.lsum / 2 + 1;  // orders n kept per point
    double2* ph = ls_smem;                               // NR
    double2* gF = ph + A.NR;                             // LS_CHUNK * nF
    double2* gaz = gF + LS_CHUNK * nF;                   // LS_CHUNK
    double2* gph = gaz + LS_CHUNK;                       // LS_CHUNK: e^{-i q.r'}
    double* gb2 = (double*)(gph + LS_CHUNK);             // LS_CHUNK
    const int T = (A.lsum + 1) * (A.lsum + 1), nmax = nF - 1;
    const int tid = threadIdx.x;
    if (A.offplane && tid == 0) {
        double w = 1.0;
        for (int j = 0; j <= A.J; ++j) {
            if (j > 0) w *= 0.5 * A.t / j;
            tw[j] = w;
        }
    }
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
                const double2 G = A.G[g], Gl = A.Glo[g];
                double qx, qy, ex, ey;
                bloch_order(kpar.x, G.x, Gl.x, qx, ex);
                bloch_order(kpar.y, G.y, Gl.y, qy, ey);
                double b2 = (qx * qx + qy * qy) / (A.k * A.k);
                // v = (q.q - k^2) / (2 eta^2 k^2), the difference compensated near a threshold
                double v = q2_minus_k2(qx, ex, qy, ey, A.k) / (2.0 * A.eta * A.eta * A.k * A.k);
                if (fabs(v) <= 1e-14) {
                    atomicExch(A.status, 9);  // on a diffraction threshold (reciprocal.rs:236-241)
                    for (int n = 0; n <= nmax; ++n) gF[tid * nF + n] = mk(0.0, 0.0);
                } else if (A.offplane) {
                    reduced_shifted(nmax, A.J, tw, v, A.eta, gF + tid * nF);
                } else {
                    reduced_limits(nmax, v, A.eta, gF + tid * nF);
                }
                gb2[tid] = b2;
                gaz[tid] = mk(qx / A.k, qy / A.k);
                double ps, pc;
                sincos(-(qx * A.sx + qy * A.sy), &ps, &pc);
                gph[tid] = mk(pc, ps);
            }
            __syncthreads();
            if (active && (even || A.offplane)) {
                const int nm = (l - am) / 2;
                const double* coef = A.coef + (size_t)lm * LS_NMAX;
                const int cnt = min(LS_CHUNK, A.NG - g0);
                for (int t = 0; t < cnt; ++t) {
                    const double b2 = gb2[t];
                    const double2* F = gF + t * nF;
                    cplx s = mk(0.0, 0.0);
                    if (A.offplane) {
                        // Horner in beta^2 over p = (l - |m| - s)/2; the orders n with n <= s <= 2n
                        const double* cz = A.coefz + (size_t)lm * LS_PMAX * LS_FMAX;
                        for (int p = (l - am) / 2; p >= 0; --p) {
                            s = cscale(s, b2);
                            const int sidx = l - am - 2 * p;
                            for (int n = (sidx + 1) / 2; n <= sidx; ++n)
                                cfma(s, mk(cz[p * LS_FMAX + n], 0.0), F[n]);
                        }
                    } else {
                        for (int n = 0; n <= nm; ++n) {  // Horner in beta^2
                            s = cscale(s, b2);
                            cfma(s, mk(coef[n], 0.0), F[n]);
                        }
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

// ---- batched periodic-array solve ----------------------------------------------------------
// One CTA per Bloch vector, X = (I - T S)^-1 T (cluster/interaction.rs:292-315 with
// sw/plan.rs:383-413 evaluate_periodic). The M x M operator (M = 2 lmax (lmax + 2), 96 at
// lmax 6) lives in registers: warp w owns the rows 8 w .. 8 w + 7 and lane l the columns
// 3 l .. 3 l + 2 of them (an 8 x 3 tile per lane; 12 warps and 168 registers a thread at
// lmax 6), assembled there from the harmonic table D / N and the plan's term lists.
//
// The inverse comes from in-place Gauss-Jordan exchange steps without row or column
// interchanges, eight rows (one warp) at a time. Block step k0: the warp owning rows
// k0..k0+7 runs the eight exchange steps on its own rows with warp collectives only (step t
// pivots on (k0 + t, p_t), p_t the not yet pivotal column with the largest |a|^2 in row
// k0 + t, ties to the lower column; with inv = 1 / a_(k0+t) p_t, u_j = a_(k0+t) j inv (j != p_t)
// and u_p = 1 + inv, the other block rows take a_rj -= a_rp u_j and row k0 + t becomes u_j,
// inv at p_t). It publishes the transformed rows U (plus 1 at each row's own pivot column) and
// p_0..p_7; after one barrier every other row takes the rank-8 update
// a_ij -= sum_t a_(i p_t) U_tj with its entries a_(i p_t) from before the update (staged per row
// in shared memory by the lanes holding them). U and the pivots are double-buffered: one barrier
// per eight rows, and a pivot warp never shares its instructions with another block's update.
// The table B then expresses the unknowns through the right-hand sides:
// (A^-1)[p_k][k'] = B[k][p_k'], so X[p_k][col] = sum_q' B[k][p_(2 lm + q')] t_lm[q'][q] for
// col = 2 lm + q (T is block diagonal per mode pair), gathered through shared memory.
// 8 M^3 real flops per Bloch vector.
constexpr int GJ_MAXM = 96;
constexpr int GJ_R = 8;  // tile rows (a warp's rows)
constexpr int GJ_C = 3;  // tile columns (a lane's columns)

__device__ __forceinline__ cplx shfl_c(cplx v, int src) {
    return mk(__shfl_sync(0xffffffffu, v.x, src), __shfl_sync(0xffffffffu, v.y, src));
}
// a[c] for a runtime c < GJ_C with static register indexing
__device__ __forceinline__ cplx pick3(const cplx* a, int c) {
    cplx v = a[0];
#pragma unroll
    for (int q = 1; q < GJ_C; ++q)
        if (c == q) v = a[q];
    return v;
}

// Entries of combo (d, s) = (4 tr + dd, j0 / 2 + ss) of A = I - T S that fall in the tile
// (rows 2d, 2d+1; columns 2s, 2s+1), unrolled by template so that the tile stays in registers.
template <int dd, int ss>
__device__ __forceinline__ void gj_assemble(cplx (&a)[GJ_R][GJ_C], const DevPlan& P, const double2* Z,
                                            const double2* __restrict__ Tm, int tr, int j0, int nlm) {
    const int d = (GJ_R / 2) * tr + dd, sidx = (j0 >> 1) + ss;
    if (d >= nlm || sidx >= nlm || 2 * sidx >= j0 + GJ_C) return;
    int lam = 1;
    while ((lam + 1) * (lam + 1) - 1 <= d) ++lam;
    const double2* t4 = Tm + (lam - 1) * 4;
    cplx Aa, Bb;
    plan_combo_sums(P, sidx * nlm + d, Z, Aa, Bb);
    const cplx cp = cadd(Aa, Bb), cn = csub(Aa, Bb);
    const double one = sidx == d ? 1.0 : 0.0;
    const cplx a00 = csub(mk(one, 0.0), cmul(t4[0], cp)), a10 = cneg(cmul(t4[2], cp)),
               a01 = cneg(cmul(t4[1], cn)), a11 = csub(mk(one, 0.0), cmul(t4[3], cn));
    const int c0 = 2 * sidx - j0;  // tile column of column 2s (-1 .. 2)
#pragma unroll
    for (int c = 0; c < GJ_C; ++c) {  // selects, not branches: the tile stays in registers
        const bool e = c == c0, o = c == c0 + 1;
        a[2 * dd][c] = e ? a00 : (o ? a01 : a[2 * dd][c]);
        a[2 * dd + 1][c] = e ? a10 : (o ? a11 : a[2 * dd + 1][c]);
    }
}

// Exchange step t of a block (rows of one warp): pivot search by two redux.sync, the pivot
// column broadcast by shuffles, 1 / a_kp = conj(a_kp) / |a_kp|^2, and the update of the
// warp's rows.
template <int t>
__device__ __forceinline__ void gj_block_step(cplx (&a)[GJ_R][GJ_C], int (&pk)[GJ_R], int bw, bool own, int j0,
                                              int M, unsigned& used, int* piv, int k0, int lane, int& s_sing) {
    pk[t] = -1;
    if (t >= bw) return;
    // pivot: largest |a|^2 (as an FP32 key, + 1 so that 0 means no candidate) over the
    // columns not yet pivotal, ties to the lower column
    unsigned key = 0u, bj = 0xffffffffu;
#pragma unroll
    for (int c = 0; c < GJ_C; ++c) {
        const int j = j0 + c;
        const unsigned kk = __float_as_uint((float)cabs2(a[t][c])) + 1u;
        if (own && j < M && !((used >> c) & 1u) && kk > key) {
            key = kk;
            bj = (unsigned)j;
        }
    }
    const unsigned kmax = __reduce_max_sync(0xffffffffu, key);
    const unsigned jmin = __reduce_min_sync(0xffffffffu, key == kmax ? bj : 0xffffffffu);
    const int p = kmax ? (int)jmin : 0, po = p / GJ_C, pc = p - po * GJ_C;
    pk[t] = p;
    cplx col[GJ_R];
#pragma unroll
    for (int r = 0; r < GJ_R; ++r) col[r] = shfl_c(pick3(a[r], pc), po);
    // an exact zero pivot (or no candidate) is singular
    const double den = cabs2(col[t]);
    if ((!(den > 0.0) || !kmax) && lane == 0) s_sing = 1;
    const double rden = __drcp_rn(den);
    const cplx inv = mk(col[t].x * rden, -col[t].y * rden);
#pragma unroll
    for (int c = 0; c < GJ_C; ++c) {
        const bool jp = j0 + c == p;
        const cplx rk = cmul(a[t][c], inv);
        const cplx u = jp ? mk(1.0 + inv.x, inv.y) : rk;
#pragma unroll
        for (int r = 0; r < GJ_R; ++r)
            if (r != t) cfma(a[r][c], cneg(col[r]), u);
        a[t][c] = jp ? inv : rk;
        if (jp) used |= 1u << c;
    }
    if (lane == 0) piv[k0 + t] = p;
}

__global__ void __launch_bounds__(384, 1) array_solve_kernel(DevPlan P, const double2* __restrict__ D,
                                                             size_t ldd, const double* __restrict__ norm,
                                                             const double2* __restrict__ Tm, int nk,
                                                             double2* __restrict__ X, int* __restrict__ status) {
    extern __shared__ double2 gj_smem[];                 // B (M x M, column-major) for the final gather
    __shared__ double2 Z[(2 * 12 + 1) * (2 * 12 + 1)];  // harmonic table, order <= 2 lmax = 12
    __shared__ double2 Ublk[2][GJ_R][GJ_MAXM];
    __shared__ double2 Ls[GJ_MAXM][GJ_R];  // each row's entries at the block's pivot columns
    __shared__ int pvt[2][GJ_R];
    __shared__ int piv[GJ_MAXM];
    __shared__ int s_sing;
    const int nlm = P.nlm, M = 2 * nlm, TR = (M + GJ_R - 1) / GJ_R, TC = (M + GJ_C - 1) / GJ_C;
    const int tid = threadIdx.x, lane = tid & 31;
    const int tr = tid >> 5, tc = lane;  // warp = tile row, lane = tile column
    const bool own = tr < TR && tc < TC;
    const bool rowwarp = tr < TR;
    const int i0 = GJ_R * tr, j0 = GJ_C * tc;
    for (int kp = blockIdx.x; kp < nk; kp += gridDim.x) {
        for (int t = tid; t < P.tsize; t += blockDim.x) Z[t] = cscale(D[(size_t)kp * ldd + t], 1.0 / norm[t]);
        if (tid == 0) s_sing = 0;
        __syncthreads();
        // A = I - T S on the tile: combo (s, d) gives rows 2d, 2d+1 of columns 2s, 2s+1; the
        // tile's rows hold d = 4 tr .. 4 tr + 3, its columns touch s = j0 / 2 and (j0 + 2) / 2
        cplx a[GJ_R][GJ_C];
#pragma unroll
        for (int r = 0; r < GJ_R; ++r)
#pragma unroll
            for (int c = 0; c < GJ_C; ++c) a[r][c] = mk(0.0, 0.0);
        if (own) {
            gj_assemble<0, 0>(a, P, Z, Tm, tr, j0, nlm);
            gj_assemble<0, 1>(a, P, Z, Tm, tr, j0, nlm);
            gj_assemble<1, 0>(a, P, Z, Tm, tr, j0, nlm);
            gj_assemble<1, 1>(a, P, Z, Tm, tr, j0, nlm);
            gj_assemble<2, 0>(a, P, Z, Tm, tr, j0, nlm);
            gj_assemble<2, 1>(a, P, Z, Tm, tr, j0, nlm);
            gj_assemble<3, 0>(a, P, Z, Tm, tr, j0, nlm);
            gj_assemble<3, 1>(a, P, Z, Tm, tr, j0, nlm);
        }
        unsigned used = 0u;  // bit c: column j0 + c is already pivotal
        bool singular = false;
        for (int kb = 0, buf = 0; GJ_R * kb < M; ++kb, buf ^= 1) {
            const int k0 = GJ_R * kb, bw = min(GJ_R, M - k0);
            if (tr == kb) {
                // the block rows: bw exchange steps inside the warp (unrolled by template so that
                // the tile stays in registers)
                int pk[GJ_R];
                gj_block_step<0>(a, pk, bw, own, j0, M, used, piv, k0, lane, s_sing);
                gj_block_step<1>(a, pk, bw, own, j0, M, used, piv, k0, lane, s_sing);
                gj_block_step<2>(a, pk, bw, own, j0, M, used, piv, k0, lane, s_sing);
                gj_block_step<3>(a, pk, bw, own, j0, M, used, piv, k0, lane, s_sing);
                gj_block_step<4>(a, pk, bw, own, j0, M, used, piv, k0, lane, s_sing);
                gj_block_step<5>(a, pk, bw, own, j0, M, used, piv, k0, lane, s_sing);
                gj_block_step<6>(a, pk, bw, own, j0, M, used, piv, k0, lane, s_sing);
                gj_block_step<7>(a, pk, bw, own, j0, M, used, piv, k0, lane, s_sing);
                // publish U (the transformed rows, plus 1 at each row's own pivot) and the pivots
                if (own) {
#pragma unroll
                    for (int t = 0; t < GJ_R; ++t)
#pragma unroll
                        for (int c = 0; c < GJ_C; ++c) {
                            const int j = j0 + c;
                            if (j >= M) continue;
                            cplx v = t < bw ? a[t][c] : mk(0.0, 0.0);
                            if (j == pk[t]) v.x += 1.0;
                            Ublk[buf][t][j] = v;
                        }
                }
                if (lane == 0)
#pragma unroll
                    for (int t = 0; t < GJ_R; ++t) pvt[buf][t] = pk[t];
            }
            __syncthreads();
            if (s_sing) {
                singular = true;
                break;
            }
            if (rowwarp && tr != kb) {
                // rank-bw update of the other rows with their entries at the pivot columns, all
                // taken before the update changes them (staged per row in shared memory by the
                // lanes that hold them)
#pragma unroll
                for (int t = 0; t < GJ_R; ++t) {
                    if (t >= bw) break;
                    const int p = pvt[buf][t];
                    if (own && p >= j0 && p < j0 + GJ_C) {
#pragma unroll
                        for (int r = 0; r < GJ_R; ++r)
                            if (i0 + r < M) Ls[i0 + r][t] = pick3(a[r], p - j0);
                        used |= 1u << (p - j0);
                    }
                }
                __syncwarp();
#pragma unroll
                for (int t = 0; t < GJ_R; ++t) {
                    if (t >= bw) break;
                    cplx nl[GJ_R];
#pragma unroll
                    for (int r = 0; r < GJ_R; ++r) nl[r] = i0 + r < M ? cneg(Ls[i0 + r][t]) : mk(0.0, 0.0);
                    if (own) {
#pragma unroll
                        for (int c = 0; c < GJ_C; ++c) {
                            const int j = j0 + c;
                            if (j >= M) continue;
                            const cplx u = Ublk[buf][t][j];
#pragma unroll
                            for (int r = 0; r < GJ_R; ++r) cfma(a[r][c], nl[r], u);
                        }
                    }
                }
            }
        }
        if (singular) {
            if (tid == 0) atomicExch(status, 5);
            __syncthreads();
            continue;
        }
        // X[p_k][col] = sum_q' B[k][p_(2 lm + q')] t_lm[q'][q], B through shared memory
        double2* Bs = gj_smem;
        if (own) {
#pragma unroll
            for (int r = 0; r < GJ_R; ++r)
#pragma unroll
                for (int c = 0; c < GJ_C; ++c)
                    if (i0 + r < M && j0 + c < M) Bs[(size_t)(j0 + c) * M + i0 + r] = a[r][c];
        }
        __syncthreads();
        double2* Xk = X + (size_t)kp * M * M;
        for (int t = tid; t < M * M; t += blockDim.x) {
            const int col = t / M, k = t - col * M;  // consecutive threads: consecutive k
            const int lm = col >> 1, q = col & 1;
            int lam = 1;
            while ((lam + 1) * (lam + 1) - 1 <= lm) ++lam;
            const double2* t4 = Tm + (lam - 1) * 4;
            cplx v = cmul(Bs[(size_t)piv[2 * lm] * M + k], t4[q]);
            cfma(v, Bs[(size_t)piv[2 * lm + 1] * M + k], t4[2 + q]);
            Xk[(size_t)col * M + piv[k]] = v;
        }
        __syncthreads();
    }
}

}  // namespace

void launch_real_table(int lsum, double k, double eta, int NR, const double2* R, double sx, double sy, double sz,
                       const double* norm, const double* reflection, double2* tab, cudaStream_t st) {
    StageScope sc(ST_LATTICE, st);
    real_table_kernel<<<(NR + 3) / 4, 128, 0, st>>>(lsum, k, eta, NR, R, sx, sy, sz, norm, reflection, tab);
}

size_t lattice_sum_smem(int lsum, int NR, bool offplane) {
    const size_t nF = offplane ? lsum + 1 : lsum / 2 + 1;
    return (size_t)NR * 16 + (size_t)LS_CHUNK * nF * 16 + 2 * LS_CHUNK * 16 + LS_CHUNK * 8;
}

void launch_lattice_sum(const LatticeSumArgs& a, int grid, cudaStream_t st) {
    StageScope sc(ST_LATTICE, st);
    size_t smem = lattice_sum_smem(a.lsum, a.NR, a.offplane != 0);
    cudaFuncSetAttribute(lattice_sum_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    lattice_sum_kernel<<<grid, 256, smem, st>>>(a);
}

void launch_array_solve(const DevPlan& P, const double2* D, size_t ldd, const double* norm, const double2* Tm, int nk,
                        double2* X, int* status, int grid, cudaStream_t st) {
    StageScope sc(ST_SMALL_LU, st);
    const int M = 2 * P.nlm;
    const int threads = 32 * ((M + GJ_R - 1) / GJ_R);  // a warp per eight rows
    const size_t smem = (size_t)M * M * sizeof(double2);
    cudaFuncSetAttribute(array_solve_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    array_solve_kernel<<<grid, threads, smem, st>>>(P, D, ldd, norm, Tm, nk, X, status);
}

}  // namespace tcu
