// 2D Ewald lattice sums of outgoing spherical waves at a complex wavenumber k (lossy embedding,
// Im k >= 0) and any shift r, with a real split eta (lattice::sum, lattice/mod.rs:283).
//
// The same split as the real-wavenumber kernels of lattice.cu (real space lattice/real.rs:149-187,
// reciprocal space lattice/reciprocal.rs:288-334 with S_lmn of reciprocal.rs:22-60 and the t-series
// of lattice/reduced.rs:223 off the plane, the self term at r' = 0), with every quantity that
// involves k complex:
//   real space   Treal_lm(rho) = -i sqrt(2/pi) (k |rho|)^l N_lm Y_lm(-rho/|rho|) I_2l(k |rho|, eta),
//                I_2l(z, eta) = eta^(2l+1)/2 sum_j c^j/j! R(l + 1/2 - j), R(d) = Gamma(d, a)/a^d at the
//                complex a = (z eta)^2/2 (special/integrals/kambe.rs:36-120). Re(k) > 0 and
//                Im(k) >= 0 with a real eta put z eta in the first quadrant, where z eta/sqrt 2 is the
//                principal root of a, so no reflected ladder arises.
//   reciprocal   F_(1/2-n)(v, 0) = Gamma(1/2-n, v)/(-v)^(1/2-n) at the complex v = (q.q/k^2 - 1)/(2 eta^2)
//                on the outgoing sheet of each diffraction order (lattice/sheets.rs): orders whose
//                k^2 - q.q lies in the near sector of the split take whole turns from the principal
//                argument, an odd number of turns adds -2 Gamma(1/2-n)/(-v)^(1/2-n), and a value
//                above the real axis changes sign (lattice/reduced.rs:18-100).
// Special functions, FP64 complex, from published methods: Gamma(d, z) for half-integer d <= 1/2
// by the power series (DLMF 8.7.3) near the origin and where Re z < 0, else by Legendre's
// continued fraction (DLMF 8.9.2, modified Lentz); R(d) for d > 1/2 by the upward recurrence
// R(d+1) = (d R(d) + e^-a)/a.
//
// Device layout as in lattice.cu: one launch tabulates Treal for the lattice points within the
// cutoff (a warp per point), one CTA per Bloch vector adds the real-space table with the Bloch
// phases and the reciprocal sum over G in chunks of 256 points (threads over G evaluate F'_n
// into shared memory, threads over lm add the chunk in a fixed order). S_lmn is evaluated as a
// polynomial in beta^2 whose coefficients (powers of -k r_z folded in) come from the host, so
// shifts on and off the plane take the same path.
#include <cuda_runtime.h>

#include "common.cuh"
#include "kernels.h"

namespace tcu {

namespace {

constexpr int CK_JMAX = 64;   // Kambe series terms
constexpr int CK_LADDER = LS_MAXL + 1 + CK_JMAX;
constexpr int CK_CHUNK = 256;  // reciprocal points per chunk
constexpr double CK_PI = 3.14159265358979323846;

__device__ __forceinline__ cplx clog_c(cplx z) { return mk(log(hypot(z.x, z.y)), atan2(z.y, z.x)); }
__device__ __forceinline__ cplx cpow_c(cplx z, double a) {  // principal z^a
    if (z.x == 0.0 && z.y == 0.0) return mk(0.0, 0.0);
    return cexpz(cscale(clog_c(z), a));
}
__device__ __forceinline__ cplx cpowi_c(cplx z, int n) {
    cplx r = mk(1.0, 0.0), b = z;
    unsigned e = (unsigned)(n < 0 ? -n : n);
    while (e) {
        if (e & 1u) r = cmul(r, b);
        b = cmul(b, b);
        e >>= 1;
    }
    return n < 0 ? cinv(r) : r;
}

// Legendre's continued fraction of Gamma(d, z) e^z z^-d (DLMF 8.9.2, even contraction), modified
// Lentz; converges off the negative real axis
__device__ cplx gamma_fraction_c(double d, cplx z) {
    const double tiny = 1e-300;
    cplx b = mk(z.x + 1.0 - d, z.y), c = mk(1.0 / tiny, 0.0), dd = cinv(b), h = dd;
    for (int i = 1; i < 2000; ++i) {
        const double an = -(double)i * ((double)i - d);
        b.x += 2.0;
        dd = cadd(cscale(dd, an), b);
        if (cabs2(dd) < 1e-300) dd = mk(tiny, 0.0);
        c = cadd(b, cscale(cinv(c), an));
        if (cabs2(c) < 1e-300) c = mk(tiny, 0.0);
        dd = cinv(dd);
        const cplx del = cmul(dd, c);
        h = cmul(h, del);
        if (fabs(del.x - 1.0) + fabs(del.y) < 1e-16) break;
    }
    return h;
}

// sum_k (-z)^k / (k! (d + k)) (DLMF 8.7.3 without its leading power)
__device__ cplx gamma_series_sum_c(double d, cplx z) {
    cplx s = mk(1.0 / d, 0.0), term = mk(1.0, 0.0);
    const double az = hypot(z.x, z.y);
    for (int k = 1; k < 600; ++k) {
        term = cscale(cmul(term, cneg(z)), 1.0 / k);
        const cplx add = cscale(term, 1.0 / (d + k));
        s = cadd(s, add);
        if (k > az && cabs2(add) < 1e-36 * cabs2(s)) break;
    }
    return s;
}

__device__ __forceinline__ bool use_fraction(cplx z) {
    const double az = hypot(z.x, z.y);
    return z.x >= 2.0 || (az >= 4.0 && z.x >= -0.3 * az);
}

// R(d) = Gamma(d, a)/a^d for half-integer d <= 1/2 and Re a > 0 (the Kambe ladder below 1/2)
__device__ cplx scaled_gamma_c(double d, cplx a) {
    if (use_fraction(a)) return cmul(cexpz(cneg(a)), gamma_fraction_c(d, a));
    return csub(cscale(cpow_c(a, -d), tgamma(d)), gamma_series_sum_c(d, a));
}

// F_(1/2-i)(v, 0) on the outgoing sheet: z = v with a zero imaginary part taken as -0 (lower side),
// g = Gamma(b, z)/(-z)^b, b = 1/2 - i; odd turns add -2 Gamma(b)/(-z)^b, Im z > 0 flips the sign
// (lattice/reduced.rs:18-100 with lattice/sheets.rs)
__device__ cplx reduced_limit_c(int i, cplx z, bool odd_turns) {
    const double b = 0.5 - i;
    // 1 / (-z)^b = (-z)^i / sqrt(-z), principal (sqrt(-z) with -z's zero imaginary part as +0);
    // formed from the positive power, it stays finite next to a threshold at large i
    const cplx mz = cneg(z);
    const cplx inv_rp = cmul(cpowi_c(mz, i), cinv(csqrt_p(mz)));
    cplx g;
    if (use_fraction(z)) {
        // Gamma(b, z) = e^-z z^b CF, and z^b / (-z)^b = e^(-+ i pi b) below / above the axis
        const double ph = (z.y > 0.0 ? 1.0 : -1.0) * CK_PI * b;
        double s, c;
        sincos(ph, &s, &c);
        g = cmul(cmul(cexpz(cneg(z)), mk(c, s)), gamma_fraction_c(b, z));
    } else {
        // Gamma(b, z) = Gamma(b) - z^b sum_k (-z)^k/(k! (b + k))
        const double ph = (z.y > 0.0 ? 1.0 : -1.0) * CK_PI * b;
        double s, c;
        sincos(ph, &s, &c);
        g = csub(cscale(inv_rp, tgamma(b)), cmul(mk(c, s), gamma_series_sum_c(b, z)));
    }
    if (odd_turns) g = csub(g, cscale(inv_rp, 2.0 * tgamma(b)));
    if (z.y > 0.0) g = cneg(g);
    return g;
}

// One warp per lattice point: Treal_lm(R) for every l <= lsum, |m| <= l, complex k.
__global__ void __launch_bounds__(128) real_table_ck_kernel(int lsum, cplx k, double eta, int NR,
                                                            const double2* __restrict__ R, double sx, double sy,
                                                            double sz, const double* __restrict__ norm,
                                                            const double* __restrict__ reflection,
                                                            double2* __restrict__ tab) {
    __shared__ cplx ladder[4][CK_LADDER];
    __shared__ cplx kam[4][LS_MAXL + 1];
    __shared__ cplx Y[4][(LS_MAXL + 1) * (LS_MAXL + 1)];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int r = blockIdx.x * 4 + warp;
    if (r >= NR) return;
    const int T = (lsum + 1) * (lsum + 1);
    const double2 p = R[r];
    double dist, u[3];
    unit_direction(-p.x - sx, -p.y - sy, -sz, dist, u);  // rho = -r' - R
    const cplx ze = cscale(k, dist * eta);
    const cplx a = cscale(cmul(ze, ze), 0.5);
    const double c = 0.5 / (eta * eta);
    // ladder[i] = R(lsum + 1/2 - i): R(1/2) and below from the series / fraction, above by recurrence
    const int nlad = lsum + 1 + CK_JMAX;
    for (int i = lsum + lane; i < nlad; i += 32) ladder[warp][i] = scaled_gamma_c(lsum + 0.5 - i, a);
    __syncwarp();
    if (lane == 0) {
        const cplx ea = cexpz(cneg(a)), ainv = cinv(a);
        cplx rr = ladder[warp][lsum];
        double d = 0.5;
        for (int i = lsum - 1; i >= 0; --i) {
            rr = cmul(cadd(cscale(rr, d), ea), ainv);
            d += 1.0;
            ladder[warp][i] = rr;
        }
    }
    if (lane <= lsum) solid_column(lsum, lane, u, reflection, Y[warp]);
    __syncwarp();
    if (lane <= lsum) {
        const int l = lane;
        cplx sum = mk(0.0, 0.0);
        double coef = 1.0;
        for (int j = 0; j < CK_JMAX; ++j) {
            if (j > 0) coef *= c / j;
            const cplx term = cscale(ladder[warp][lsum - l + j], coef);
            sum = cadd(sum, term);
            if (j > c + 3.0 && cabs2(term) <= 1e-34 * cabs2(sum)) break;
        }
        kam[warp][l] = cscale(sum, 0.5 * pow(eta, 2 * l + 1));
    }
    __syncwarp();
    const double s2p = 0.79788456080286535588;  // sqrt(2/pi)
    const cplx kd = cscale(k, dist);
    for (int lm = lane; lm < T; lm += 32) {
        int l = (int)sqrt((double)lm);
        while (l * l > lm) --l;
        while ((l + 1) * (l + 1) <= lm) ++l;
        const cplx f = cscale(cmul(cpowi_c(kd, l), kam[warp][l]), s2p * norm[lm]);
        const cplx fy = cmul(f, Y[warp][lm]);
        tab[(size_t)r * T + lm] = mk(fy.y, -fy.x);  // -i f y
    }
}

// F'_n = (2 eta^2)^n / (sqrt 2 eta) sum_j tw[j] F_(1/2-n-j)(v, 0), n = 0..nmax, tw[j] = (t/2)^j / j!
__device__ void reduced_shifted_c(int nmax, int J, const cplx* tw, cplx v, bool odd_turns, double eta, cplx* out) {
    for (int n = 0; n <= nmax; ++n) out[n] = mk(0.0, 0.0);
    for (int i = 0; i <= nmax + J; ++i) {
        const cplx L = reduced_limit_c(i, v, odd_turns);
        for (int n = min(nmax, i); n >= max(0, i - J); --n) cfma(out[n], tw[i - n], L);
    }
    double factor = 1.0 / (1.4142135623730950488 * eta);
    const double step = 2.0 * eta * eta;
    for (int n = 0; n <= nmax; ++n) {
        out[n] = cscale(out[n], factor);
        factor *= step;
    }
}

// Whole turns of v on the outgoing sheet of an order (lattice/sheets.rs): orders whose k^2 - q.q
// lies in the near sector of the split (|arg| of (k eta)^2 + 1/2 < pi/2) follow arg(k^2 - q.q);
// the others stay on the principal sheet. Returns whether the number of turns is odd.
__device__ bool odd_turns_of(const LatticeSumCkArgs& A, double q2, cplx v) {
    const cplx sq = mk(A.ksq.x - q2, A.ksq.y);
    const bool near = sq.x > 0.0 && sq.y * sq.y <= A.near * sq.x * sq.x;
    if (A.has_near && !near) return false;
    double turn;
    if (sq.y == 0.0) {
        turn = sq.x > 0.0 ? 0.0 : CK_PI;
    } else {
        turn = atan2(sq.y, sq.x);
        if (turn < 0.0) turn += 2.0 * CK_PI;
    }
    const double sheet = turn - CK_PI - A.turn;
    const double turns = rint((sheet - atan2(v.y, v.x)) / (2.0 * CK_PI));
    return fmod(fabs(turns), 2.0) == 1.0;
}

// One CTA per Bloch vector (complex k).
__global__ void __launch_bounds__(256) lattice_sum_ck_kernel(LatticeSumCkArgs A) {
    extern __shared__ double2 ck_smem[];
    __shared__ cplx tw[LS_TMAX + 1];
    const int nF = A.lsum + 1;
    double2* ph = ck_smem;                    // NR
    double2* gF = ph + A.NR;                  // CK_CHUNK * nF
    double2* gq = gF + CK_CHUNK * nF;         // CK_CHUNK: (q_x, q_y)
    double2* gph = gq + CK_CHUNK;             // CK_CHUNK: e^{-i q.r'}
    double2* gb2 = gph + CK_CHUNK;            // CK_CHUNK: beta^2 = q.q / k^2
    const int T = (A.lsum + 1) * (A.lsum + 1), nmax = A.lsum;
    const int tid = threadIdx.x;
    if (tid == 0) {
        cplx w = mk(1.0, 0.0);
        const cplx half_t = cscale(A.t, 0.5);
        for (int j = 0; j <= A.J; ++j) {
            if (j > 0) w = cscale(cmul(w, half_t), 1.0 / j);
            tw[j] = w;
        }
    }
    const cplx kinv = cinv(A.k), kinv2 = cmul(kinv, kinv);
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
        const bool active = lm < T;
        if (active) {
            while ((l + 1) * (l + 1) <= lm) ++l;
            m = lm - l * l - l;
        }
        const int am = m < 0 ? -m : m;
        cplx acc = mk(0.0, 0.0);
        if (active)
            for (int r = 0; r < A.NR; ++r) cfma(acc, __ldg(&A.realtab[(size_t)r * T + lm]), ph[r]);
        cplx rec = mk(0.0, 0.0);
        for (int g0 = 0; g0 < A.NG; g0 += CK_CHUNK) {
            __syncthreads();
            const int g = g0 + tid;
            if (tid < CK_CHUNK && g < A.NG) {
                const double2 G = A.G[g], Gl = A.Glo[g];
                double qx, qy, ex, ey;
                bloch_order(kpar.x, G.x, Gl.x, qx, ex);
                bloch_order(kpar.y, G.y, Gl.y, qy, ey);
                const double q2 = qx * qx + qy * qy;
                const cplx b2 = cscale(kinv2, q2);
                // v = (q.q - k^2) / (2 eta^2 k^2): Re(q.q - k^2) = (q.q - Re(k)^2) + Im(k)^2 compensated
                const cplx d = mk(q2_minus_k2(qx, ex, qy, ey, A.k.x) + A.k.y * A.k.y, -2.0 * A.k.x * A.k.y);
                cplx v = cscale(cmul(d, kinv2), 1.0 / (2.0 * A.eta * A.eta));
                if (v.y == 0.0) v.y = -0.0;  // lower side (lattice/sheets.rs:12-17)
                if (hypot(v.x, v.y) <= 1e-14) {
                    atomicExch(A.status, 9);  // on a diffraction threshold (reciprocal.rs:236-241)
                    for (int n = 0; n <= nmax; ++n) gF[tid * nF + n] = mk(0.0, 0.0);
                } else {
                    reduced_shifted_c(nmax, A.J, tw, v, odd_turns_of(A, q2, v), A.eta, gF + tid * nF);
                }
                gb2[tid] = b2;
                gq[tid] = mk(qx, qy);
                double ps, pc;
                sincos(-(qx * A.sx + qy * A.sy), &ps, &pc);
                gph[tid] = mk(pc, ps);
            }
            __syncthreads();
            if (active) {
                const cplx* cz = A.coef + (size_t)lm * LS_PMAX * LS_FMAX;
                const int cnt = min(CK_CHUNK, A.NG - g0);
                for (int t = 0; t < cnt; ++t) {
                    const cplx b2 = gb2[t];
                    const double2* F = gF + t * nF;
                    cplx s = mk(0.0, 0.0);
                    // Horner in beta^2 over p = (l - |m| - s)/2; the orders n with n <= s <= 2n
                    for (int p = (l - am) / 2; p >= 0; --p) {
                        s = cmul(s, b2);
                        const int sidx = l - am - 2 * p;
                        for (int n = (sidx + 1) / 2; n <= sidx; ++n) cfma(s, cz[p * LS_FMAX + n], F[n]);
                    }
                    const double2 q = gq[t];
                    const cplx az = cmul(mk(q.x, m < 0 ? -q.y : q.y), kinv);  // (q_x +- i q_y)/k
                    cfma(rec, s, cmul(cpowi_c(az, am), gph[t]));
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

}  // namespace

void launch_real_table_ck(int lsum, cplx k, double eta, int NR, const double2* R, double sx, double sy, double sz,
                          const double* norm, const double* reflection, double2* tab, cudaStream_t st) {
    StageScope sc(ST_LATTICE, st);
    real_table_ck_kernel<<<(NR + 3) / 4, 128, 0, st>>>(lsum, k, eta, NR, R, sx, sy, sz, norm, reflection, tab);
}

size_t lattice_sum_ck_smem(int lsum, int NR) {
    return (size_t)NR * 16 + (size_t)CK_CHUNK * (lsum + 1) * 16 + 3 * CK_CHUNK * 16;
}

void launch_lattice_sum_ck(const LatticeSumCkArgs& a, int grid, cudaStream_t st) {
    StageScope sc(ST_LATTICE, st);
    const size_t smem = lattice_sum_ck_smem(a.lsum, a.NR);
    cudaFuncSetAttribute(lattice_sum_ck_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    lattice_sum_ck_kernel<<<grid, 256, smem, st>>>(a);
}

}  // namespace tcu
