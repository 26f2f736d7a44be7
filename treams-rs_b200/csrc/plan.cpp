// Host-side construction of the geometry-independent translation plan: for every source
// (l, m) and destination (lambda, mu) of a block, the degree terms (p, weight) of the
// same-helicity coefficient A and the cross coefficient B. Built once per lmax and kept
// on the device; the kernels combine them with h_p(kr) Y_p^(m-mu) per sphere pair.
//
// The weights follow the coupling of treams-rs sw/coupling.rs:86-123 (tl_vsw_A / tl_vsw_B
// of treams): pref = (-1)^m / 2 sqrt((2l+1)(2lambda+1) / (l(l+1) lambda(lambda+1))) times
//   A: (l(l+1) + lambda(lambda+1) - p(p+1)) (2p+1) i^(lambda-l+p) sqrt((p-(m-mu))!/(p+(m-mu))!)
//      (l lambda p; m -mu mu-m) (l lambda p; 0 0 0),        p = l+lambda, l+lambda-2, ...
//   B: sqrt((l+lambda+1+p)(l+lambda+1-p)(p+lambda-l)(p-lambda+l)) (2p+1) i^(lambda-l+p)
//      sqrt(...) (l lambda p; m -mu mu-m) (l lambda p-1; 0 0 0),  p = l+lambda-1, ...
// down to max(|l-lambda| (+1 for B), |m-mu|) (coupling.rs:146-160). The Wigner 3j symbols
// here come from Racah's closed formula evaluated in binary128, exact to far below double
// rounding for the degrees a plan uses (<= 2 * 10), instead of the reference's recurrence.
#include <cmath>
#include <cstdint>
#include <vector>

#include "plan.h"

namespace tcu {

typedef __float128 q128;

static q128 qfact(int n) {
    q128 f = 1;
    for (int i = 2; i <= n; ++i) f *= i;
    return f;
}

// Racah's formula for (j1 j2 j3; m1 m2 m3)
double wigner3j_racah(int j1, int j2, int j3, int m1, int m2, int m3) {
    if (m1 + m2 + m3 != 0 || j3 < std::abs(j1 - j2) || j3 > j1 + j2 || std::abs(m1) > j1 || std::abs(m2) > j2 ||
        std::abs(m3) > j3 || j1 < 0 || j2 < 0 || j3 < 0)
        return 0.0;
    int tmin = std::max(0, std::max(j2 - j3 - m1, j1 - j3 + m2));
    int tmax = std::min(j1 + j2 - j3, std::min(j1 - m1, j2 + m2));
    q128 sum = 0;
    for (int t = tmin; t <= tmax; ++t) {
        q128 den = qfact(t) * qfact(j3 - j2 + t + m1) * qfact(j3 - j1 + t - m2) * qfact(j1 + j2 - j3 - t) *
                   qfact(j1 - t - m1) * qfact(j2 - t + m2);
        q128 term = 1 / den;
        sum += (t % 2 == 0) ? term : -term;
    }
    q128 delta = qfact(j1 + j2 - j3) * qfact(j1 - j2 + j3) * qfact(-j1 + j2 + j3) / qfact(j1 + j2 + j3 + 1);
    q128 f = qfact(j1 + m1) * qfact(j1 - m1) * qfact(j2 + m2) * qfact(j2 - m2) * qfact(j3 + m3) * qfact(j3 - m3);
    long double root = sqrtl((long double)(delta * f));
    int ph = j1 - j2 - m3;
    long double v = (long double)sum * root;
    if (((ph % 2) + 2) % 2 == 1) v = -v;
    return (double)v;
}

static void ipow(int n, double& re, double& im) {
    switch (((n % 4) + 4) % 4) {
        case 0: re = 1; im = 0; break;
        case 1: re = 0; im = 1; break;
        case 2: re = -1; im = 0; break;
        default: re = 0; im = -1; break;
    }
}

// sqrt((p-q)!/(p+q)!) in binary128
static double fact_ratio_sqrt(int p, int q) {
    long double r = (long double)(qfact(p - q) / qfact(p + q));
    return (double)sqrtl(r);
}

HostPlan build_plan(int L) {
    HostPlan plan;
    plan.L = L;
    plan.nlm = L * (L + 2);
    plan.order = 2 * L;
    int nlm = plan.nlm;
    std::vector<int> ls(nlm), ms(nlm);
    for (int l = 1, i = 0; l <= L; ++l)
        for (int m = -l; m <= l; ++m, ++i) {
            ls[i] = l;
            ms[i] = m;
        }
    plan.combo.resize((size_t)nlm * nlm * 2);
    for (int s = 0; s < nlm; ++s) {
        int l = ls[s], m = ms[s];
        for (int d = 0; d < nlm; ++d) {
            int lam = ls[d], mu = ms[d];
            int c = s * nlm + d;
            int start = (int)plan.idx.size();
            double pref = 0.5 * ((m % 2 == 0) ? 1.0 : -1.0) *
                          std::sqrt(double((2 * l + 1) * (2 * lam + 1)) / (double(l * (l + 1)) * double(lam * (lam + 1))));
            int counts[2] = {0, 0};
            for (int cross = 0; cross < 2; ++cross) {
                int pstart = l + lam - cross;
                int pend = std::max(std::abs(lam - l) + cross, std::abs(m - mu));
                for (int p = pstart; p >= pend; p -= 2) {
                    double factor = cross ? std::sqrt(double(l + lam + 1 + p) * double(l + lam + 1 - p) *
                                                      double(p + lam - l) * double(p - lam + l))
                                          : double(l * (l + 1) + lam * (lam + 1) - p * (p + 1));
                    int q = p - cross;
                    double w1 = wigner3j_racah(l, lam, p, m, -mu, mu - m);
                    double w0 = wigner3j_racah(l, lam, q, 0, 0, 0);
                    double mag = pref * factor * double(2 * p + 1) * fact_ratio_sqrt(p, m - mu) * w1 * w0;
                    double re, im;
                    ipow(lam - l + p, re, im);
                    if (mag * mag * (re * re + im * im) > 0.0) {
                        plan.idx.push_back((uint16_t)(p * p + p + m - mu));
                        plan.w.push_back(mag * re);
                        plan.w.push_back(mag * im);
                        counts[cross] += 1;
                    }
                }
            }
            plan.combo[2 * c] = start;
            plan.combo[2 * c + 1] = counts[0] | (counts[1] << 16);
        }
    }
    int T = (plan.order + 1) * (plan.order + 1);
    plan.reflection.resize(T);
    for (int p = 0; p <= plan.order; ++p)
        for (int m = -p; m <= p; ++m) {
            int a = std::abs(m);
            long double r = (long double)(qfact(p - a) / qfact(p + a));
            plan.reflection[p * p + p + m] = (double)(((a % 2) ? -1.0L : 1.0L) * r);
        }
    return plan;
}

}  // namespace tcu
