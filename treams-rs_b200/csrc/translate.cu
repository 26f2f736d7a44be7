// Per-entry vector spherical wave translation coefficients at complex polar arguments
// (kr, theta, phi), the elementwise form of sw.translate (python/treams_rs/sw.py:70,
// treams-core sw/polar.rs:163-251). One thread per element: the radial sequence z_p(kr)
// and the associated Legendre column P_p^|q|(cos theta) of the element's single order
// q = m - mu are built in registers, then the plan's A and B term lists of the mode pair are
// summed. Helicity modes: A + (2 pol - 1) B for equal helicities, 0 otherwise; parity modes:
// A for equal and B for different parities (sw/coupling.rs:127-140).
#include <cuda_runtime.h>

#include "common.cuh"
#include "kernels.h"
#include "plan.h"

namespace tcu {

namespace {

constexpr int TR_MAXP = 21;  // term degrees p <= l + lambda <= 20

// Outgoing h_0..h_last(z) at complex z != 0. |z| >= 0.5: upward recurrence of h itself from
// h_-1 = e^{iz}/z, h_0 = -i e^{iz}/z (DLMF 10.49.6, 10.51.1; stable, h is the dominant
// solution), which keeps the decaying combination for Im z > 0. Below: j_p by its power
// series (DLMF 10.53.1) plus y_p by the upward recurrence from y_-1 = sin z/z, y_0 = -cos z/z.
__device__ void chankel_seq(int last, cplx z, cplx* h) {
    const cplx inv = cinv(z);
    if (sqrt(cabs2(z)) >= 0.5) {
        cplx e = cexpz(mk(-z.y, z.x));  // e^{iz}
        cplx prev = cmul(e, inv), cur = cmul(mk(e.y, -e.x), inv);
        for (int p = 0; p <= last; ++p) {
            h[p] = cur;
            cplx next = csub(cscale(cmul(inv, cur), double(2 * p + 1)), prev);
            prev = cur;
            cur = next;
        }
        return;
    }
    const cplx sq = cmul(z, z);
    cplx zl = mk(1.0, 0.0);
    double df = 1.0;
    cplx yprev = cmul(csin(z), inv), ycur = cneg(cmul(ccos(z), inv));
    for (int p = 0; p <= last; ++p) {
        if (p > 0) {
            zl = cmul(zl, z);
            df *= double(2 * p + 1);
        }
        cplx term = cscale(zl, 1.0 / df), sum = term;
        for (int q = 1; q < 24; ++q) {
            term = cscale(cmul(term, sq), -1.0 / (2.0 * q * (2.0 * (p + q) + 1.0)));
            sum = cadd(sum, term);
        }
        h[p] = mk(sum.x - ycur.y, sum.y + ycur.x);  // j + i y
        cplx ynext = csub(cscale(cmul(inv, ycur), double(2 * p + 1)), yprev);
        yprev = ycur;
        ycur = ynext;
    }
}

// Regular j_0..j_last(z) at complex z: power series below |z| = 0.5, else Miller's backward
// recurrence from order last + 24 + 2|z| normalised by j_0 = sin z / z or j_1.
__device__ void cbessel_seq(int last, cplx z, cplx* j) {
    const double az = sqrt(cabs2(z));
    if (az < 0.5) {
        const cplx sq = cmul(z, z);
        cplx zl = mk(1.0, 0.0);
        double df = 1.0;
        for (int p = 0; p <= last; ++p) {
            if (p > 0) {
                zl = cmul(zl, z);
                df *= double(2 * p + 1);
            }
            cplx term = cscale(zl, 1.0 / df), sum = term;
            for (int q = 1; q < 24; ++q) {
                term = cscale(cmul(term, sq), -1.0 / (2.0 * q * (2.0 * (p + q) + 1.0)));
                sum = cadd(sum, term);
            }
            j[p] = sum;
        }
        return;
    }
    const cplx inv = cinv(z);
    const int start = last + 24 + (int)(2.0 * az);
    cplx fnext = mk(0.0, 0.0), f = mk(1e-200, 0.0);
    for (int p = 0; p <= last; ++p) j[p] = mk(0.0, 0.0);
    for (int k = start; k >= 1; --k) {
        cplx fprev = csub(cscale(cmul(inv, f), double(2 * k + 1)), fnext);
        fnext = f;
        f = fprev;
        if (cabs2(f) > 1e300) {
            f = cscale(f, 1e-150);
            fnext = cscale(fnext, 1e-150);
            for (int p = 0; p <= last; ++p) j[p] = cscale(j[p], 1e-150);
        }
        if (k - 1 <= last) j[k - 1] = f;
        if (k <= last) j[k] = fnext;
    }
    const cplx s = csin(z), c = ccos(z);
    const cplx j0 = cmul(s, inv), j1 = csub(cmul(s, cmul(inv, inv)), cmul(c, inv));
    const cplx scale = cabs2(j0) >= cabs2(j1) ? cdiv(j0, j[0]) : cdiv(j1, j[1]);
    for (int p = 0; p <= last; ++p) j[p] = cmul(j[p], scale);
}

__global__ void translate_kernel(DevPlan P, size_t count, const int* __restrict__ labels, const cplx* __restrict__ args,
                                 bool helicity, bool singular, cplx* __restrict__ out) {
    const size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= count) return;
    const int* lb = labels + 6 * e;
    const int lam = lb[0], mu = lb[1], pol = lb[2], l = lb[3], m = lb[4], qol = lb[5];
    const cplx kr = args[3 * e], th = args[3 * e + 1], ph = args[3 * e + 2];
    if (helicity && pol != qol) {
        out[e] = mk(0.0, 0.0);
        return;
    }
    if (singular && sqrt(cabs2(kr)) < 1e-16) {  // the self term is zero (sw/polar.rs:150-160)
        out[e] = mk(0.0, 0.0);
        return;
    }
    const int q = m - mu, aq = q < 0 ? -q : q, last = l + lam;
    cplx rad[TR_MAXP];
    if (singular)
        chankel_seq(last, kr, rad);
    else
        cbessel_seq(last, kr, rad);
    // P_p^|q|(cos theta) for p = |q|..last with sin theta taken directly (no sqrt(1 - cos^2),
    // which loses the coupling at tiny angles): P_|q|^|q| = (-1)^|q| (2|q|-1)!! sin^|q|,
    // P_{p}^|q| = ((2p-1) x P_{p-1} - (p+|q|-1) P_{p-2}) / (p-|q|) (DLMF 14.10.3)
    const cplx x = ccos(th), sn = csin(th);
    cplx leg[TR_MAXP];
    cplx diag = mk(1.0, 0.0);
    for (int k = 1; k <= aq; ++k) diag = cscale(cmul(diag, sn), -double(2 * k - 1));
    cplx pcur = diag, pprev = mk(0.0, 0.0);
    for (int p = aq; p <= last; ++p) {
        if (p > aq) {
            cplx next = cscale(csub(cscale(cmul(x, pcur), double(2 * p - 1)), cscale(pprev, double(p + aq - 1))),
                               1.0 / double(p - aq));
            pprev = pcur;
            pcur = next;
        }
        leg[p] = pcur;
    }
    // e^{i q phi}; negative orders carry (-1)^|q| (p-|q|)!/(p+|q|)! (the plan's reflection)
    const cplx eq = cexpz(mk(-q * ph.y, q * ph.x));
    const int s = l * l - 1 + l + m, d = lam * lam - 1 + lam + mu;
    const int2 cb = __ldg(&P.combo[s * P.nlm + d]);
    int t = cb.x;
    const int na = cb.y & 0xffff, nb = cb.y >> 16;
    cplx A = mk(0.0, 0.0), B = mk(0.0, 0.0);
    for (int k = 0; k < na + nb; ++k, ++t) {
        const int idx = __ldg(&P.idx[t]);
        const int pq = idx - q;  // p (p + 1)
        int p = (int)sqrt((double)pq);
        while (p * (p + 1) > pq) --p;
        while ((p + 1) * (p + 2) <= pq) ++p;
        cplx zp = cmul(rad[p], leg[p]);
        if (q < 0) zp = cscale(zp, P.reflection[idx]);
        const cplx w = __ldg(&P.w[t]);
        if (k < na)
            cfma(A, w, zp);
        else
            cfma(B, w, zp);
    }
    A = cmul(A, eq);
    B = cmul(B, eq);
    cplx v;
    if (helicity)
        v = pol ? cadd(A, B) : csub(A, B);
    else
        v = pol == qol ? A : B;
    out[e] = v;
}

}  // namespace

void launch_translate(const DevPlan& P, size_t count, const int* labels, const cplx* args, bool helicity,
                      bool singular, cplx* out, cudaStream_t st) {
    if (!count) return;
    translate_kernel<<<(unsigned)((count + 127) / 128), 128, 0, st>>>(P, count, labels, args, helicity, singular, out);
}

}  // namespace tcu
