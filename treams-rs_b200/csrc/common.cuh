// Shared device helpers: complex arithmetic on double2/float2, the radial and angular
// special functions of the translation coefficients, and small launch utilities.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#define TCU_HD __host__ __device__ __forceinline__

typedef double2 cplx;

TCU_HD cplx mk(double r, double i) { return make_double2(r, i); }
TCU_HD cplx cadd(cplx a, cplx b) { return mk(a.x + b.x, a.y + b.y); }
TCU_HD cplx csub(cplx a, cplx b) { return mk(a.x - b.x, a.y - b.y); }
TCU_HD cplx cmul(cplx a, cplx b) { return mk(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x); }
TCU_HD cplx cscale(cplx a, double s) { return mk(a.x * s, a.y * s); }
TCU_HD cplx cconj(cplx a) { return mk(a.x, -a.y); }
TCU_HD cplx cneg(cplx a) { return mk(-a.x, -a.y); }
// a += b * c
TCU_HD void cfma(cplx& a, cplx b, cplx c) {
    a.x = fma(b.x, c.x, fma(-b.y, c.y, a.x));
    a.y = fma(b.x, c.y, fma(b.y, c.x, a.y));
}
// a += conj(b) * c
TCU_HD void cfma_conj(cplx& a, cplx b, cplx c) {
    a.x = fma(b.x, c.x, fma(b.y, c.y, a.x));
    a.y = fma(b.x, c.y, fma(-b.y, c.x, a.y));
}
TCU_HD double cabs2(cplx a) { return a.x * a.x + a.y * a.y; }
TCU_HD cplx cdiv(cplx a, cplx b) {
    // Smith's algorithm
    if (fabs(b.x) >= fabs(b.y)) {
        double r = b.y / b.x, d = b.x + b.y * r;
        return mk((a.x + a.y * r) / d, (a.y - a.x * r) / d);
    } else {
        double r = b.x / b.y, d = b.x * r + b.y;
        return mk((a.x * r + a.y) / d, (a.y * r - a.x) / d);
    }
}
TCU_HD cplx cinv(cplx b) { return cdiv(mk(1.0, 0.0), b); }
TCU_HD cplx cexp_i(double x) {  // e^{ix}
    double s, c;
    sincos(x, &s, &c);
    return mk(c, s);
}
TCU_HD cplx csqrt_p(cplx z) {  // principal square root
    double r = hypot(z.x, z.y);
    if (r == 0.0) return mk(0.0, 0.0);
    double t = sqrt(0.5 * (r + fabs(z.x)));
    if (z.x >= 0.0) return mk(t, z.y / (2.0 * t));
    return mk(fabs(z.y) / (2.0 * t), copysign(t, z.y));
}
TCU_HD cplx csin(cplx z) {
    double s, c;
    sincos(z.x, &s, &c);
    return mk(s * cosh(z.y), c * sinh(z.y));
}
TCU_HD cplx ccos(cplx z) {
    double s, c;
    sincos(z.x, &s, &c);
    return mk(c * cosh(z.y), -s * sinh(z.y));
}
TCU_HD cplx cexpz(cplx z) {
    double e = exp(z.x), s, c;
    sincos(z.y, &s, &c);
    return mk(e * c, e * s);
}

// q.q - k^2 for real q = (qx + ex, qy + ey) (ex, ey: small low parts) and k, with the products
// and the sums compensated (error-free transformations: fma for the products, two-sum for the
// additions): next to a diffraction threshold q.q and k^2 agree in most digits, and the plain
// difference loses them.
__device__ __forceinline__ double q2_minus_k2(double qx, double ex, double qy, double ey, double k) {
    const double p1 = qx * qx, e1 = fma(qx, qx, -p1);
    const double p2 = qy * qy, e2 = fma(qy, qy, -p2);
    const double p3 = k * k, e3 = fma(k, k, -p3);
    const double s1 = p1 + p2, z1 = s1 - p1, t1 = (p1 - (s1 - z1)) + (p2 - z1);
    const double s2 = s1 - p3, z2 = s2 - s1, t2 = (s1 - (s2 - z2)) + (-p3 - z2);
    return s2 + ((((t1 + t2) + (e1 + e2)) - e3) + 2.0 * (qx * ex + qy * ey));
}
// q = kpar + G with G = Gh + Gl a reciprocal vector kept to twice the FP64 precision: the rounded
// component and the low part (the rounding error of the sum plus Gl)
__device__ __forceinline__ void bloch_order(double kp, double gh, double gl, double& q, double& e) {
    q = kp + gh;
    const double z = q - kp;
    e = ((kp - (q - z)) + (gh - z)) + gl;
}

// ---- radial functions -----------------------------------------------------------------
// Outgoing spherical Hankel functions h_0..h_last at real x > 0. For 0.5 <= x <= 1e4 the
// upward recurrence h_{p+1} = (2p+1)/x h_p - h_{p-1} from h_-1 = e^{ix}/x, h_0 = -i e^{ix}/x
// (DLMF 10.49.6, 10.51.1); below 0.5 the regular part j_p comes from its power series
// (DLMF 10.53.1) and the irregular y_p from the same upward recurrence, which is stable
// for the dominant solution.
template <int MAXP>
__device__ __forceinline__ void series_j_real(int last, double x, double* j) {
    // j_p(x) = x^p / (2p+1)!! * sum_q (-x^2/2)^q / (q! (2p+3)(2p+5)...(2p+2q+1))
    double lead = 1.0;
    for (int p = 0; p <= last && p < MAXP; ++p) {
        if (p > 0) lead *= x / double(2 * p + 1);
        double term = lead, sum = lead, sq = x * x;
        for (int q = 1; q < 24; ++q) {
            term *= -sq / (2.0 * q * (2.0 * (p + q) + 1.0));
            sum += term;
        }
        j[p] = sum;
    }
}
template <int MAXP>
__device__ __forceinline__ void hankel_sequence(int last, double x, cplx* h) {
    double inv = 1.0 / x, s, c;
    sincos(x, &s, &c);
    if (x >= 0.5) {
        cplx prev = mk(c * inv, s * inv), cur = mk(s * inv, -c * inv);
        for (int p = 0; p <= last; ++p) {
            h[p] = cur;
            cplx next = mk(double(2 * p + 1) * inv * cur.x - prev.x, double(2 * p + 1) * inv * cur.y - prev.y);
            prev = cur;
            cur = next;
        }
        return;
    }
    double j[MAXP];
    series_j_real<MAXP>(last, x, j);
    double yprev = s * inv, ycur = -c * inv;  // y_-1, y_0
    for (int p = 0; p <= last; ++p) {
        h[p] = mk(j[p], ycur);
        double ynext = double(2 * p + 1) * inv * ycur - yprev;
        yprev = ycur;
        ycur = ynext;
    }
}
// Regular spherical Bessel j_0..j_last at real x >= 0: series below 0.5, else Miller's
// backward recurrence from order last + 20 + 2x normalised by j_0 or j_1.
template <int MAXP>
__device__ __forceinline__ void bessel_j_sequence(int last, double x, double* j) {
    if (x < 0.5) {
        series_j_real<MAXP>(last, x, j);
        return;
    }
    int start = last + 24 + int(2.0 * x);
    double fnext = 0.0, f = 1e-200, inv = 1.0 / x;
    double keep[MAXP];
    for (int q = 0; q < MAXP; ++q) keep[q] = 0.0;
    for (int k = start; k >= 1; --k) {
        double fprev = double(2 * k + 1) * inv * f - fnext;
        fnext = f;
        f = fprev;
        if (fabs(f) > 1e200) {
            f *= 1e-200;
            fnext *= 1e-200;
            for (int q = 0; q < MAXP; ++q) keep[q] *= 1e-200;
        }
        if (k - 1 <= last && k - 1 < MAXP) keep[k - 1] = f;
        if (k <= last && k < MAXP) keep[k] = fnext;
    }
    double s, c;
    sincos(x, &s, &c);
    double j0 = s * inv, j1 = s * inv * inv - c * inv;
    double scale = (fabs(j0) >= fabs(j1)) ? j0 / keep[0] : j1 / keep[1];
    for (int p = 0; p <= last && p < MAXP; ++p) j[p] = keep[p] * scale;
}

// Solid harmonics r^p P_p^m(cos theta) e^{i m phi} at a unit vector for p <= order, table
// index p*p+p+m: the diagonal P_m^m from the ladder factor -(2m-1)(x + i y), then the
// degree recurrence P_{p} = ((2p-1) z P_{p-1} - (p+m-1) r^2 P_{p-2}) / (p-m) (DLMF 14.10.3
// in solid form); negative orders by P_p^{-m} e^{-i m phi} = (-1)^m (p-m)!/(p+m)! conj(.).
// `reflection[idx]` holds those factors for every table entry. One thread computes one
// order column: this is the work of lane `m` of a warp.
__device__ __forceinline__ void solid_column(int order, int m, const double* u, const double* reflection, cplx* table) {
    cplx xy = mk(u[0], u[1]);
    double z = u[2], r2 = u[0] * u[0] + u[1] * u[1] + u[2] * u[2];
    cplx diag = mk(1.0, 0.0);
    for (int k = 1; k <= m; ++k) diag = cscale(cmul(diag, xy), -double(2 * k - 1));
    cplx p = diag, prev = mk(0.0, 0.0);
    for (int deg = m; deg <= order; ++deg) {
        if (deg > m) {
            double a = double(2 * deg - 1) / double(deg - m);
            double b = double(deg + m - 1) / double(deg - m);
            cplx next = mk(a * z * p.x - b * r2 * prev.x, a * z * p.y - b * r2 * prev.y);
            prev = p;
            p = next;
        }
        table[deg * deg + deg + m] = p;
        if (m > 0) {
            int idx = deg * deg + deg - m;
            table[idx] = cscale(cconj(p), reflection[idx]);
        }
    }
}

// Length and direction of a displacement, scaled by its largest component first.
TCU_HD bool unit_direction(double x, double y, double zc, double& r, double* u) {
    double scale = fmax(fabs(x), fmax(fabs(y), fabs(zc)));
    if (scale < 2.2250738585072014e-308) return false;
    double a = x / scale, b = y / scale, c = zc / scale;
    double norm = sqrt(a * a + b * b + c * c);
    r = scale * norm;
    u[0] = a / norm;
    u[1] = b / norm;
    u[2] = c / norm;
    return true;
}
