// CPU ORACLE — TEST INFRASTRUCTURE ONLY.
//
// A plain C++17 restatement of the treams-rs (yaugenst/treams-rs) FP64 algorithms on the
// cluster multiple-scattering hot path. Only the tests, the smoke check and the CPU-baseline
// leg of the benchmark load this library, and only to check or time the CUDA library;
// the product path never calls it. Each function names the reference file:line it follows.
//
// Third-party numerics the reference takes from crates (not vendored in the reference tree):
//   complex-bessel 0.3.0 (AMOS)  -> complex j_l by series below |z| = 0.5 and Miller's
//                                   backward recurrence above it; h_l by the upward
//                                   recurrence from h_0, h_-1 (DLMF 10.51.1); the real-argument
//                                   h_l below x = 0.5 as j_l (series) + i y_l (upward).
//   faer 0.24.4 (LU)             -> right-looking partial-pivot LU (max |z| pivot).
//   libm lgamma                  -> std::lgamma.
#include <algorithm>
#include <cmath>
#include <complex>
#include <cstdint>
#include <cstring>
#include <map>
#include <utility>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

using cd = std::complex<double>;
static const cd I1(0.0, 1.0);

// ---------------------------------------------------------------------------------------
// special/mod.rs:104-120 — log factorial cache and sqrt((l-m)!/(l+m)!)
static double log_factorial(int n) {
    static std::vector<double> cache = [] {
        std::vector<double> v(257);
        for (int i = 0; i <= 256; ++i) v[i] = std::lgamma(double(i) + 1.0);
        return v;
    }();
    if (n >= 0 && n <= 256) return cache[n];
    return std::lgamma(double(n) + 1.0);
}
static double factorial_ratio_sqrt(int l, int m) {
    return std::exp(0.5 * (log_factorial(l - m) - log_factorial(l + m)));
}
static double parity(int n) { return (n % 2 == 0) ? 1.0 : -1.0; }
static cd cpowi(cd z, int n) {  // integer power by repeated products (num_complex powi)
    if (n < 0) return cd(1.0, 0.0) / cpowi(z, -n);
    cd r(1.0, 0.0);
    for (int i = 0; i < n; ++i) r *= z;
    return r;
}
static cd ipow(int n) {  // i^n for any integer n
    int r = ((n % 4) + 4) % 4;
    switch (r) {
        case 0: return cd(1, 0);
        case 1: return cd(0, 1);
        case 2: return cd(-1, 0);
        default: return cd(0, -1);
    }
}

// ---------------------------------------------------------------------------------------
// special/wigner.rs:36-317 — Wigner 3j rows by the two-sided Schulten-Gordon recurrence
static double w_c(int j1, int j2, int j3, int m3) {
    double a = double(j3) * j3 - double(j1 - j2) * (j1 - j2);
    double b = double(j1 + j2 + 1) * (j1 + j2 + 1) - double(j3) * j3;
    double c = double(j3) * j3 - double(m3) * m3;
    return std::sqrt(a * b * c);
}
static double w_d(int j1, int j2, int j3, int m1, int m2, int m3) {
    return double(2 * j3 + 1) *
           (double(j3 * (j3 + 1)) * double(m2 - m1) + double(j2 * (j2 + 1) - j1 * (j1 + 1)) * double(m3));
}
static double initial_j(int j1, int j2, int m1, int m2) {
    return parity(j1 + m1) *
           std::exp(0.5 * (log_factorial(j1 - m1) + log_factorial(j1 + m1) + log_factorial(2 * j1 - 2 * j2) +
                           log_factorial(2 * j2) - log_factorial(j2 - m2) - log_factorial(j2 + m2) -
                           log_factorial(j1 - j2 - m1 - m2) - log_factorial(j1 - j2 + m1 + m2) -
                           log_factorial(2 * j1 + 1)));
}
static double initial_m(int j1, int j2, int m1, int m2) {
    return parity(j2 + m2) *
           std::exp(0.5 * (log_factorial(j1 + m1) + log_factorial(j2 + m2) + log_factorial(j1 + j2 - m1 - m2) +
                           log_factorial(2 * m1 + 2 * m2) - log_factorial(j1 - m1) - log_factorial(j2 - m2) -
                           log_factorial(j1 - j2 + m1 + m2) - log_factorial(j2 - j1 + m1 + m2) -
                           log_factorial(j1 + j2 + m1 + m2 + 1)));
}
static double lowest(int j1, int j2, int m1, int m2, int minimum) {
    if (minimum == j1 - j2) return initial_j(j1, j2, m1, m2);
    if (minimum == j2 - j1) return initial_j(j2, j1, m2, m1);
    if (minimum == m1 + m2) return initial_m(j1, j2, m1, m2);
    return initial_m(j2, j1, -m2, -m1);
}
static double highest(int j1, int j2, int m1, int m2) {
    int maximum = j1 + j2, m3 = -m1 - m2;
    return parity(maximum - m3) *
           std::exp(0.5 * (log_factorial(2 * j1) + log_factorial(2 * j2) + log_factorial(maximum + m3) +
                           log_factorial(maximum - m3) - log_factorial(2 * maximum + 1) - log_factorial(j1 - m1) -
                           log_factorial(j1 + m1) - log_factorial(j2 - m2) - log_factorial(j2 + m2)));
}
static int growth_end(int j1, int j2, int m1, int m2, int minimum, int stop) {
    int m3 = -m1 - m2;
    double ratio = INFINITY;
    for (int j = minimum + 1; j <= stop; ++j) {
        if (minimum == 0 && j == 1)
            ratio = -double(m2 - m1) / w_c(j1, j2, 1, m3);
        else
            ratio = (-w_d(j1, j2, j - 1, m1, m2, m3) - double(j) * w_c(j1, j2, j - 1, m3) / ratio) /
                    (double(j - 1) * w_c(j1, j2, j, m3));
        if (std::fabs(ratio) < 1.0) return j;
    }
    return stop + 1;
}
static int decay_start(int j1, int j2, int m1, int m2, int maximum, int stop) {
    int m3 = -m1 - m2;
    double ratio = INFINITY;
    for (int j = maximum - 1; j >= stop; --j) {
        if (j == maximum - 1)
            ratio = -w_d(j1, j2, maximum, m1, m2, m3) / (double(maximum + 1) * w_c(j1, j2, maximum, m3));
        else
            ratio = (-w_d(j1, j2, j + 1, m1, m2, m3) - double(j + 1) * w_c(j1, j2, j + 2, m3) / ratio) /
                    (double(j + 2) * w_c(j1, j2, j + 1, m3));
        if (std::fabs(ratio) < 1.0) return j + 1;
    }
    return stop;
}
static int turn_of(int j1, int j2, int m1, int m2, int minimum, int maximum, int first, int last) {
    int sw = (j1 + j2 - std::abs(j1 - j2)) / 4 + std::abs(j1 - j2);
    int ge = growth_end(j1, j2, m1, m2, minimum, last);
    if (ge > last) return last + 1;
    int bound = std::max(ge, first);
    if (sw <= bound) return bound;
    return std::min(sw, decay_start(j1, j2, m1, m2, maximum, bound));
}
template <class F>
static void w_visit(int j1, int j2, int m1, int m2, int first, int last, F emit) {
    int m3 = -m1 - m2;
    int minimum = std::max(std::abs(j1 - j2), std::abs(m3));
    int maximum = j1 + j2;
    int turn = turn_of(j1, j2, m1, m2, minimum, maximum, first, last);
    if (first < turn) {
        double value = lowest(j1, j2, m1, m2, minimum), previous = 0.0;
        for (int j = minimum; j < std::min(turn, last + 1); ++j) {
            if (j > minimum) {
                double next;
                if (minimum == 0 && j == 1)
                    next = -value * double(m2 - m1) / w_c(j1, j2, 1, m3);
                else
                    next = (-w_d(j1, j2, j - 1, m1, m2, m3) * value - double(j) * w_c(j1, j2, j - 1, m3) * previous) /
                           (double(j - 1) * w_c(j1, j2, j, m3));
                previous = value;
                value = next;
            }
            if (j >= first) emit(j, value);
        }
    }
    if (turn > last) return;
    double value = highest(j1, j2, m1, m2), previous = 0.0;
    if (last == maximum) emit(maximum, value);
    for (int j = maximum - 1; j >= std::max(turn, first); --j) {
        double next;
        if (j == maximum - 1)
            next = -w_d(j1, j2, j + 1, m1, m2, m3) * value / (double(j + 2) * w_c(j1, j2, j + 1, m3));
        else
            next = (-w_d(j1, j2, j + 1, m1, m2, m3) * value - double(j + 1) * w_c(j1, j2, j + 2, m3) * previous) /
                   (double(j + 2) * w_c(j1, j2, j + 1, m3));
        previous = value;
        value = next;
        if (j <= last) emit(j, value);
    }
}
struct W3jRow {
    int first = 0;
    std::vector<double> values;
    W3jRow() {}
    W3jRow(int j1, int j2, int m1, int m2) {
        if (j1 < 0 || j2 < 0 || std::abs(m1) > j1 || std::abs(m2) > j2) return;
        first = std::max(std::abs(j1 - j2), std::abs(m1 + m2));
        int len = j1 + j2 + 1 - first;
        if (len <= 0) return;
        values.assign(len, 0.0);
        w_visit(j1, j2, m1, m2, first, j1 + j2, [&](int j3, double v) {
            int i = j3 - first;
            if (i >= 0 && i < (int)values.size()) values[i] = v;
        });
    }
    double get(int j3) const {
        int i = j3 - first;
        if (i < 0 || i >= (int)values.size()) return 0.0;
        return values[i];
    }
};
static double wigner3j(int j1, int j2, int j3, int m1, int m2, int m3) {
    if (j1 < 0 || j2 < 0 || j3 < 0 || j3 < std::abs(j1 - j2) || j3 > j1 + j2 || std::abs(m1) > j1 ||
        std::abs(m2) > j2 || std::abs(m3) > j3 || m1 + m2 + m3 != 0)
        return 0.0;
    double s = 0.0;
    w_visit(j1, j2, m1, m2, j3, j3, [&](int, double v) { s = v; });
    return s;
}

// ---------------------------------------------------------------------------------------
// sw/mod.rs:114-125 — modes: l ascending, m = -l..l, pol 1 before pol 0
struct Mode { int l, m, pol; };
static std::vector<Mode> modes(int lmax) {
    std::vector<Mode> out;
    for (int l = 1; l <= lmax; ++l)
        for (int m = -l; m <= l; ++m) {
            out.push_back({l, m, 1});
            out.push_back({l, m, 0});
        }
    return out;
}

// ---------------------------------------------------------------------------------------
// sw/coupling.rs:19-168 — degree terms of the A (same) and B (cross) coefficients
static void degrees(int l, int m, int lambda, int mu, bool cross, std::vector<int>& out) {
    out.clear();
    int start = l + lambda - (cross ? 1 : 0);
    int end = std::max(std::abs(lambda - l) + (cross ? 1 : 0), std::abs(m - mu));
    int count = std::max(start - end + 2, 0) / 2;
    for (int k = 0; k < count; ++k) out.push_back(start - 2 * k);
}
static cd tl_vsw_term(int l, int m, int lambda, int mu, int p, int q, const W3jRow& r0, const W3jRow& r1) {
    if (p < std::max(std::abs(m + mu), std::abs(l - lambda)) || p > l + lambda || q < std::abs(l - lambda) ||
        q > l + lambda || (q + l + lambda) % 2 != 0)
        return cd(0, 0);
    return double(2 * p + 1) * ipow(lambda - l + p) * factorial_ratio_sqrt(p, m + mu) * r0.get(p) * r1.get(q);
}
struct Coupling {
    std::vector<std::pair<int, cd>> same, cross;
};
static Coupling coupling_new(int l, int m, int lambda, int mu, const W3jRow& zeros) {
    Coupling c;
    W3jRow orders(l, lambda, m, -mu);
    double sign = (m % 2 == 0) ? 1.0 : -1.0;
    double pref = 0.5 * sign *
                  std::sqrt(double((2 * l + 1) * (2 * lambda + 1)) / (double(l * (l + 1)) * double(lambda * (lambda + 1))));
    std::vector<int> ps;
    for (int cr = 0; cr < 2; ++cr) {
        degrees(l, m, lambda, mu, cr == 1, ps);
        for (int p : ps) {
            double factor;
            if (cr)
                factor = std::sqrt(double(l + lambda + 1 + p) * double(l + lambda + 1 - p) * double(p + lambda - l) *
                                   double(p - lambda + l));
            else
                factor = double(l * (l + 1) + lambda * (lambda + 1) - p * (p + 1));
            cd w = pref * factor * tl_vsw_term(l, m, lambda, -mu, p, p - cr, orders, zeros);
            if (std::norm(w) > 0.0) (cr ? c.cross : c.same).push_back({p, w});
        }
    }
    return c;
}

// ---------------------------------------------------------------------------------------
// sw/plan.rs:71-203 — TranslationPlan::between (helicity) and evaluate_table
struct Term { int index; cd weight; };
struct Plan {
    int M = 0, lmax = 0;          // modes per block, largest harmonic degree
    std::vector<int> starts;      // M*M + 1, column-major entries (source outer)
    std::vector<Term> terms;
};
static Plan plan_between(int L, bool helicity) {
    Plan plan;
    std::vector<Mode> md = modes(L);
    int M = (int)md.size();
    plan.M = M;
    plan.lmax = 2 * L;
    std::map<std::pair<int, int>, W3jRow> zeros;
    for (int l = 1; l <= L; ++l)
        for (int lam = 1; lam <= L; ++lam) zeros[{l, lam}] = W3jRow(l, lam, 0, 0);
    std::map<std::pair<std::pair<int, int>, std::pair<int, int>>, Coupling> cache;
    plan.starts.push_back(0);
    for (int s = 0; s < M; ++s) {
        const Mode& from = md[s];
        for (int d = 0; d < M; ++d) {
            const Mode& to = md[d];
            bool equal = to.pol == from.pol;
            bool same = helicity ? equal : equal;
            bool cross = helicity ? equal : !equal;
            if (same || cross) {
                auto key = std::make_pair(std::make_pair(from.l, from.m), std::make_pair(to.l, to.m));
                auto it = cache.find(key);
                if (it == cache.end())
                    it = cache.emplace(key, coupling_new(from.l, from.m, to.l, to.m, zeros[{from.l, to.l}])).first;
                const Coupling& c = it->second;
                double sgn = helicity ? (2.0 * from.pol - 1.0) : 1.0;
                if (same)
                    for (auto& t : c.same) plan.terms.push_back({t.first * t.first + t.first + from.m - to.m, t.second});
                if (cross)
                    for (auto& t : c.cross)
                        plan.terms.push_back({t.first * t.first + t.first + from.m - to.m, sgn * t.second});
            }
            plan.starts.push_back((int)plan.terms.size());
        }
    }
    return plan;
}
static void plan_evaluate_table(const Plan& plan, const cd* table, cd* out) {
    int E = plan.M * plan.M;
    for (int e = 0; e < E; ++e) {
        cd s(0, 0);
        for (int t = plan.starts[e]; t < plan.starts[e + 1]; ++t) s += plan.terms[t].weight * table[plan.terms[t].index];
        out[e] = s;
    }
}

// ---------------------------------------------------------------------------------------
// special/harmonics.rs:108-116 direction; :147-305 SolidTable::visit (values only)
static bool direction(const double* x, double& r, double unit[3]) {
    double scale = std::max(std::fabs(x[0]), std::max(std::fabs(x[1]), std::fabs(x[2])));
    if (scale < 2.2250738585072014e-308) return false;
    double s[3] = {x[0] / scale, x[1] / scale, x[2] / scale};
    double norm = std::sqrt(s[0] * s[0] + s[1] * s[1] + s[2] * s[2]);
    r = scale * norm;
    for (int i = 0; i < 3; ++i) unit[i] = s[i] / norm;
    return true;
}
// table[p*p+p+m] = r^p P_p^m(z/r) e^{i m phi} for p <= order
static void solid_table(int order, const double pos[3], cd* table) {
    double x = pos[0], y = pos[1], z = pos[2];
    double r2 = x * x + y * y + z * z;
    cd xy(x, y);
    cd diagonal(1.0, 0.0);
    for (int o = 0; o <= order; ++o) {
        if (o > 0) diagonal *= -double(2 * o - 1) * xy;
        cd p = diagonal, prev(0, 0);
        for (int deg = o; deg <= order; ++deg) {
            if (deg > o) {
                double a = double(2 * deg - 1) / double(deg - o);
                double b = double(deg + o - 1) / double(deg - o);
                cd next = a * z * p - b * r2 * prev;
                prev = p;
                p = next;
            }
            table[deg * deg + deg + o] = p;
            if (o > 0) {
                double refl = parity(o) * std::exp(log_factorial(deg - o) - log_factorial(deg + o));
                table[deg * deg + deg - o] = refl * std::conj(p);
            }
        }
    }
}

// ---------------------------------------------------------------------------------------
// Spherical Bessel functions.
// special/bessel.rs:495-522 — h_p(x), real x in [0.5, 1e4], last <= 64: upward recurrence
// from h_-1 = e^{ix}/x, h_0 = -i e^{ix}/x. Other real x > 0: j_p by its power series
// (bessel.rs:425-432 for |x| < 0.5) or backward recurrence, y_p by upward recurrence.
static cd sph_j_series(int l, cd z) {
    // j_l(z) = sum_q (-z^2/2)^q z^l / (q! (2l+2q+1)!!), bessel.rs:425-432, 30 terms
    double df = 1.0;
    for (int i = 0; i <= l; ++i) df *= double(2 * i + 1);
    cd term = cpowi(z, l) / df;
    cd sum = term, sq = z * z;
    for (int q = 1; q < 30; ++q) {
        term *= -sq / (2.0 * q * (2.0 * (l + q) + 1.0));
        sum += term;
    }
    return sum;
}
// j_0..j_lmax at complex z (|z| >= 0.5) by Miller's backward recurrence normalised by
// j_0 = sin z / z (or j_1 where |j_0| is smaller).
static void sph_j_sequence(int lmax, cd z, cd* out) {
    if (std::abs(z) < 0.5) {
        for (int l = 0; l <= lmax; ++l) out[l] = sph_j_series(l, z);
        return;
    }
    int start = lmax + 20 + (int)(std::abs(z) * 1.5) + 10;
    std::vector<cd> f(start + 2);
    f[start + 1] = 0.0;
    f[start] = 1e-30;
    for (int k = start; k >= 1; --k) {
        f[k - 1] = double(2 * k + 1) / z * f[k] - f[k + 1];
        if (std::abs(f[k - 1]) > 1e250) {  // rescale
            for (int q = k - 1; q <= start + 1; ++q) f[q] *= 1e-250;
        }
    }
    cd j0 = std::sin(z) / z;
    cd j1 = std::sin(z) / (z * z) - std::cos(z) / z;
    cd scale = (std::abs(j0) >= std::abs(j1)) ? j0 / f[0] : j1 / f[1];
    for (int l = 0; l <= lmax; ++l) out[l] = f[l] * scale;
}
// h_0..h_last at complex z != 0: upward recurrence of y_l plus j_l from the sequence above
static void sph_h_sequence(int last, cd z, cd* out) {
    std::vector<cd> j(last + 1);
    sph_j_sequence(last, z, j.data());
    cd y0 = -std::cos(z) / z;
    cd ym1 = std::sin(z) / z;  // y_{-1}
    cd prev = ym1, cur = y0;
    for (int l = 0; l <= last; ++l) {
        out[l] = j[l] + I1 * cur;
        cd next = double(2 * l + 1) / z * cur - prev;
        prev = cur;
        cur = next;
    }
}
static void spherical_hankels(int last, double x, cd* out) {
    if (last <= 64 && x >= 0.5 && x <= 1e4) {
        double inv = 1.0 / x, s = std::sin(x), c = std::cos(x);
        cd previous(c * inv, s * inv), current(s * inv, -c * inv);
        for (int d = 0; d <= last; ++d) {
            out[d] = current;
            if (d < last) {
                cd next = (double(2 * d + 1) * inv) * current - previous;
                previous = current;
                current = next;
            }
        }
        return;
    }
    sph_h_sequence(last, cd(x, 0.0), out);
}
static void spherical_bessels_j(int last, double x, cd* out) { sph_j_sequence(last, cd(x, 0.0), out); }

// Radial jet (value, first, second) from the next order, bessel.rs:152-160
struct Jet3 { cd value, first, second; };
static Jet3 jet_from_next_order(double order, cd z, cd value, cd next) {
    Jet3 j;
    j.value = value;
    j.first = order * value / z - next;
    j.second = -2.0 * j.first / z + order * (order + 1.0) * (value / z) / z - value;
    return j;
}
static Jet3 spherical_radial(int l, cd z, bool singular) {
    if (!singular && std::abs(z) < 0.5) {
        // series jets: value and derivatives from the series (bessel.rs:370-400)
        double df = 1.0;
        for (int i = 0; i <= l; ++i) df *= double(2 * i + 1);
        double lead = 1.0 / df;
        Jet3 term;
        term.value = lead * cpowi(z, l);
        term.first = l > 0 ? lead * double(l) * cpowi(z, l - 1) : cd(0, 0);
        term.second = l > 1 ? lead * double(l * (l - 1)) * cpowi(z, l - 2) : cd(0, 0);
        Jet3 sum = term;
        cd sq = z * z;
        for (int q = 1; q < 30; ++q) {
            double f = -1.0 / (2.0 * q * (2.0 * (l + q) + 1.0));
            Jet3 nt;
            nt.value = f * sq * term.value;
            nt.first = f * (sq * term.first + 2.0 * z * term.value);
            nt.second = f * (sq * term.second + 4.0 * z * term.first + 2.0 * term.value);
            term = nt;
            sum.value += term.value;
            sum.first += term.first;
            sum.second += term.second;
        }
        return sum;
    }
    std::vector<cd> seq(l + 2);
    if (singular)
        sph_h_sequence(l + 1, z, seq.data());
    else
        sph_j_sequence(l + 1, z, seq.data());
    return jet_from_next_order(double(l), z, seq[l], seq[l + 1]);
}

// ---------------------------------------------------------------------------------------
// coeffs/mie.rs:18-38 (Riccati), :133-185 (interface), :190-206 (inverse2), :209-251 (mie)
// for a homogeneous nonmagnetic achiral sphere (epsilon inside, vacuum outside);
// coeffs/material.rs:50-70 (index sqrt(eps mu), impedance sqrt(mu/eps)).
struct Riccati { cd waves[2][2]; };  // [kind][0: f, 1: f' + f/x]
static Riccati riccati_new(int l, cd x) {
    Riccati r;
    for (int kind = 0; kind < 2; ++kind) {
        Jet3 f = spherical_radial(l, x, kind == 1);
        r.waves[kind][0] = f.value;
        r.waves[kind][1] = f.first + f.value / x;
    }
    return r;
}
// out[4] = 2x2 Mie matrix in helicity order (negative, positive), row-major
static void mie_sphere(int l, double size, cd eps, cd* out) {
    cd n_in = std::sqrt(eps), n_out(1.0, 0.0);
    cd z_in = std::sqrt(cd(1.0, 0.0) / eps), z_out(1.0, 0.0);
    cd x[2][2] = {{size * n_in, size * n_in}, {size * n_out, size * n_out}};
    cd zz[2] = {z_in, z_out};
    Riccati rad[2][2];
    for (int side = 0; side < 2; ++side) {
        rad[side][0] = riccati_new(l, x[side][0]);
        rad[side][1] = rad[side][0];  // achiral: both helicities share one argument
    }
    cd f[4][4];
    cd ratio = zz[1] / zz[0];
    for (int p = 0; p < 2; ++p) {
        cd square = x[1][p] * x[1][p];
        for (int q = 0; q < 2; ++q) {
            double sign = (p == q) ? 1.0 : -1.0;
            cd a = (ratio + sign) / (2.0 * I1);
            cd factor = a * square;
            for (int kind = 0; kind < 2; ++kind) {
                const cd* inner = rad[0][q].waves[kind];
                for (int ok = 0; ok < 2; ++ok) {
                    const cd* outer = rad[1][p].waves[1 - ok];
                    double os = (ok == 0) ? 1.0 : -1.0;
                    cd term = os * (outer[1] * inner[0] - sign * outer[0] * inner[1]);
                    f[p + ok * 2][q + kind * 2] = term * factor;
                }
            }
        }
    }
    // q = f * [I; 0] (one interface)
    cd qm[4][2];
    for (int i = 0; i < 4; ++i)
        for (int j = 0; j < 2; ++j) qm[i][j] = f[i][j];
    // inverse2 of the upper 2x2, scaled
    double scale = 0.0;
    for (int i = 0; i < 2; ++i)
        for (int j = 0; j < 2; ++j) scale = std::max(scale, std::max(std::fabs(qm[i][j].real()), std::fabs(qm[i][j].imag())));
    cd a00 = qm[0][0] / scale, a01 = qm[0][1] / scale, a10 = qm[1][0] / scale, a11 = qm[1][1] / scale;
    cd det = a00 * a11 - a01 * a10;
    cd inv[2][2] = {{a11 / det / scale, -a01 / det / scale}, {-a10 / det / scale, a00 / det / scale}};
    for (int i = 0; i < 2; ++i)
        for (int j = 0; j < 2; ++j) out[i * 2 + j] = qm[2 + i][0] * inv[0][j] + qm[2 + i][1] * inv[1][j];
}
// tmatrix/sphere.rs:43-80 + coeffs/mie.rs:123-130 — 2x2 block per degree in mode order
// (pol 1 first): [[v11, v10], [v01, v00]], row-major.
static void mie_block_mode_order(int l, double size, cd eps, cd* out) {
    cd v[4];
    mie_sphere(l, size, eps, v);
    out[0] = v[3];
    out[1] = v[2];
    out[2] = v[1];
    out[3] = v[0];
}

// ---------------------------------------------------------------------------------------
// Plan evaluation at a displacement: sw/plan.rs:224-289 (values + evaluate_table)
static void plan_evaluate(const Plan& plan, double k, const double pos[3], bool singular, cd* out) {
    int T = (plan.lmax + 1) * (plan.lmax + 1);
    std::vector<cd> table(T, cd(0, 0));
    double r, unit[3];
    if (!direction(pos, r, unit)) {
        if (!singular) table[0] = cd(1.0, 0.0);
        plan_evaluate_table(plan, table.data(), out);
        return;
    }
    std::vector<cd> rad(plan.lmax + 1), Y(T);
    if (singular)
        spherical_hankels(plan.lmax, k * r, rad.data());
    else
        spherical_bessels_j(plan.lmax, k * r, rad.data());
    solid_table(plan.lmax, unit, Y.data());
    for (int p = 0; p <= plan.lmax; ++p)
        for (int m = -p; m <= p; ++m) table[p * p + p + m] = rad[p] * Y[p * p + p + m];
    plan_evaluate_table(plan, table.data(), out);
}

// ---------------------------------------------------------------------------------------
// pw/expand.rs:23-66 (spherical_prefactor, spherical_coefficient), special/legendre.rs:26-122
// (legendre_factors, angular_jets, polarized_angular), pw/field.rs:20-26 (phase)
static void legendre_factors(int max, int m, cd z, std::vector<cd>& vals) {  // vals[l - |m|]
    vals.clear();
    int order = std::abs(m);
    if (max < order) return;
    cd p(1.0, 0.0);
    if (m >= 0)
        for (int k = 1; k <= m; ++k) p *= -double(2 * k - 1);
    else
        for (int k = 1; k <= -m; ++k) p *= 1.0 / double(2 * k);
    vals.push_back(p);
    if (max == order) return;
    cd prev = p;
    p *= (double(2 * order + 1) / double(order - m + 1)) * z;
    vals.push_back(p);
    for (int k = order + 2; k <= max; ++k) {
        cd next = (double(2 * k - 1) * z * p - double(k + m - 1) * prev) * (1.0 / double(k - m));
        prev = p;
        p = next;
        vals.push_back(p);
    }
}
static cd legendre_factor(int l, int m, cd z) {
    std::vector<cd> v;
    legendre_factors(l, m, z, v);
    if (v.empty()) return cd(0, 0);
    return v.back();
}
static cd polarized_angular_helicity(int l, int m, cd cosine, cd sine, int pol) {
    cd pi(0, 0), tau(0, 0);
    if (m == 0) {
        tau = sine * legendre_factor(l, 1, cosine);
    } else {
        std::vector<cd> v;
        legendre_factors(l, m, cosine, v);
        cd upper = v.empty() ? cd(0, 0) : v.back();
        cd lower = v.size() >= 2 ? v[v.size() - 2] : cd(0, 0);
        cd power = (std::abs(m) - 1 == 0) ? cd(1, 0) : cpowi(sine, std::abs(m) - 1);
        pi = double(m) * power * upper;
        tau = power * (double(l) * cosine * upper - double(l + m) * lower);
    }
    return tau + (2.0 * pol - 1.0) * pi;
}
static cd pw_to_sw(const Mode& mode, const cd kvec[3], int pol) {
    if (mode.pol != pol) return cd(0, 0);
    int l = mode.l, m = mode.m;
    cd pref = 2.0 * std::sqrt(M_PI * double(2 * l + 1) / double(l * (l + 1))) * factorial_ratio_sqrt(l, m) * ipow(l);
    cd transverse(0, 0), xy[2] = {0.0, 0.0};
    if (kvec[0] != 0.0 || kvec[1] != 0.0) {
        transverse = std::sqrt(kvec[0] * kvec[0] + kvec[1] * kvec[1]);
        xy[0] = kvec[0] / transverse;
        xy[1] = kvec[1] / transverse;
    }
    cd k = std::sqrt(kvec[0] * kvec[0] + kvec[1] * kvec[1] + kvec[2] * kvec[2]);
    bool axis = transverse == cd(0, 0);
    cd azimuth = axis ? cd(1, 0) : cpowi(xy[0] - I1 * xy[1], m);
    cd cosine = axis ? cd(((kvec[2] / k).real() >= 0.0) ? 1.0 : -1.0, 0.0) : kvec[2] / k;
    cd sine = transverse / k;
    return pref * azimuth * polarized_angular_helicity(l, m, cosine, sine, pol);
}
static cd pw_phase(const cd kvec[3], const double* point) {
    double angle = kvec[0].real() * point[0] + kvec[1].real() * point[1] + kvec[2].real() * point[2];
    double att = kvec[0].imag() * point[0] + kvec[1].imag() * point[1] + kvec[2].imag() * point[2];
    double s = std::exp(-att);
    return cd(s * std::cos(angle), s * std::sin(angle));
}

// ---------------------------------------------------------------------------------------
// linalg/mod.rs:398-428 (Lu::new) with faer's partial-pivot LU semantics; equilibration is
// applied as in linalg/mod.rs:137-310 only when the spread test requires it.
struct LuFactor {
    int n = 0;
    std::vector<cd> a;        // packed L\U, column-major
    std::vector<int> piv;     // row swapped with row k at step k
    std::vector<double> row, col;  // equilibration scales (empty = none)
};
static bool needs_equilibration(const std::vector<cd>& A, int n) {
    double mn = INFINITY, mx = 0.0;
    for (auto& z : A) {
        double mag = std::max(std::fabs(z.real()), std::fabs(z.imag()));
        if (mag > 0) mn = std::min(mn, mag);
        mx = std::max(mx, mag);
    }
    if (mx > 0.0) {
        if (mn / mx >= 0.1) return false;
        bool diag_ok = true;
        for (int i = 0; i < n; ++i) {
            cd z = A[(size_t)i * n + i];
            if (std::max(std::fabs(z.real()), std::fabs(z.imag())) / mx < 0.1) { diag_ok = false; break; }
        }
        if (diag_ok) return false;
    }
    return true;
}
static int lu_factor(LuFactor& f) {
    int n = f.n;
    std::vector<cd>& a = f.a;
    f.piv.assign(n, 0);
    if (needs_equilibration(a, n)) {
        // row/column max scaling (linalg/mod.rs:166-209, xGEEQU); Sinkhorn balancing omitted
        f.row.assign(n, 0.0);
        f.col.assign(n, 0.0);
        for (int j = 0; j < n; ++j)
            for (int i = 0; i < n; ++i) {
                cd z = a[(size_t)j * n + i];
                f.row[i] = std::max(f.row[i], std::max(std::fabs(z.real()), std::fabs(z.imag())));
            }
        for (int i = 0; i < n; ++i) {
            if (f.row[i] == 0.0) return 3;
            f.row[i] = 1.0 / f.row[i];
        }
        for (int j = 0; j < n; ++j) {
            double cm = 0.0;
            for (int i = 0; i < n; ++i) {
                a[(size_t)j * n + i] *= f.row[i];
                cd z = a[(size_t)j * n + i];
                cm = std::max(cm, std::max(std::fabs(z.real()), std::fabs(z.imag())));
            }
            if (cm == 0.0) return 3;
            f.col[j] = 1.0 / cm;
            for (int i = 0; i < n; ++i) a[(size_t)j * n + i] *= f.col[j];
        }
    }
    const int nb = 64;
    for (int k0 = 0; k0 < n; k0 += nb) {
        int kb = std::min(nb, n - k0);
        // panel factorization with row swaps applied across all columns
        for (int k = k0; k < k0 + kb; ++k) {
            int p = k;
            double best = std::abs(a[(size_t)k * n + k]);
            for (int i = k + 1; i < n; ++i) {
                double v = std::abs(a[(size_t)k * n + i]);
                if (v > best) { best = v; p = i; }
            }
            f.piv[k] = p;
            if (best == 0.0) return 3;
            if (p != k)
                for (int j = 0; j < n; ++j) std::swap(a[(size_t)j * n + k], a[(size_t)j * n + p]);
            cd inv = 1.0 / a[(size_t)k * n + k];
            for (int i = k + 1; i < n; ++i) a[(size_t)k * n + i] *= inv;
            for (int j = k + 1; j < k0 + kb; ++j) {
                cd u = a[(size_t)j * n + k];
                if (u == cd(0, 0)) continue;
                cd* cj = &a[(size_t)j * n];
                const cd* ck = &a[(size_t)k * n];
                for (int i = k + 1; i < n; ++i) cj[i] -= ck[i] * u;
            }
        }
        int rest = n - (k0 + kb);
        if (rest <= 0) continue;
        // U12 = L11^{-1} A12
        #pragma omp parallel for schedule(static)
        for (int j = k0 + kb; j < n; ++j) {
            cd* cj = &a[(size_t)j * n];
            for (int k = k0; k < k0 + kb; ++k) {
                cd u = cj[k];
                const cd* ck = &a[(size_t)k * n];
                for (int i = k + 1; i < k0 + kb; ++i) cj[i] -= ck[i] * u;
            }
        }
        // A22 -= L21 U12
        #pragma omp parallel for schedule(static)
        for (int j = k0 + kb; j < n; ++j) {
            cd* cj = &a[(size_t)j * n];
            for (int k = k0; k < k0 + kb; ++k) {
                cd u = cj[k];
                if (u == cd(0, 0)) continue;
                const cd* ck = &a[(size_t)k * n];
                for (int i = k0 + kb; i < n; ++i) cj[i] -= ck[i] * u;
            }
        }
    }
    for (int i = 0; i < n; ++i)
        if (a[(size_t)i * n + i] == cd(0, 0)) return 3;
    return 0;
}
static void lu_solve(const LuFactor& f, cd* b, int nrhs) {
    int n = f.n;
    const std::vector<cd>& a = f.a;
    for (int c = 0; c < nrhs; ++c) {
        cd* x = b + (size_t)c * n;
        if (!f.row.empty())
            for (int i = 0; i < n; ++i) x[i] *= f.row[i];
        for (int k = 0; k < n; ++k)
            if (f.piv[k] != k) std::swap(x[k], x[f.piv[k]]);
        for (int k = 0; k < n; ++k) {
            cd xk = x[k];
            const cd* ck = &a[(size_t)k * n];
            for (int i = k + 1; i < n; ++i) x[i] -= ck[i] * xk;
        }
        for (int k = n - 1; k >= 0; --k) {
            const cd* ck = &a[(size_t)k * n];
            x[k] /= ck[k];
            cd xk = x[k];
            for (int i = 0; i < k; ++i) x[i] -= ck[i] * xk;
        }
        if (!f.col.empty())
            for (int i = 0; i < n; ++i) x[i] *= f.col[i];
    }
}

// ---------------------------------------------------------------------------------------
// linalg/gmres.rs:119-347 — restarted GMRES, two MGS passes, Givens, true residual
static double vnorm(const cd* v, size_t n) {
    double s = 0.0;
    for (size_t i = 0; i < n; ++i) s = std::hypot(s, std::abs(v[i]));
    return s;
}
template <class Apply>
static int gmres_solve(size_t n, const cd* rhs, cd* answer, double rtol, double atol, int restart_opt, int max_iter,
                       Apply apply, int* iterations_out, double* residual_out) {
    int restart = std::min<long long>(std::min<long long>(restart_opt, (long long)n), max_iter);
    std::vector<cd> residual(rhs, rhs + n);
    std::fill(answer, answer + n, cd(0, 0));
    double rhs_norm = vnorm(rhs, n);
    double tol = std::max(atol, rtol * rhs_norm);
    int iterations = 0;
    std::vector<std::vector<cd>> basis;
    std::vector<cd> h((restart + 1) * restart), g(restart + 1), w(n), prod(n);
    std::vector<std::pair<double, cd>> rot;
    while (true) {
        double rn = vnorm(residual.data(), n);
        *residual_out = rn;
        *iterations_out = iterations;
        if (std::isfinite(rn) && rn <= tol) return 0;
        if (!std::isfinite(rn) || iterations >= max_iter) return 4;
        basis.clear();
        basis.emplace_back(n);
        for (size_t i = 0; i < n; ++i) basis[0][i] = residual[i] / rn;
        std::fill(h.begin(), h.end(), cd(0, 0));
        std::fill(g.begin(), g.end(), cd(0, 0));
        g[0] = rn;
        rot.clear();
        int used = 0;
        for (int j = 0; j < restart; ++j) {
            apply(basis[j].data(), w.data());
            for (int pass = 0; pass < 2; ++pass)
                for (int i = 0; i <= j; ++i) {
                    cd dot(0, 0);
                    for (size_t q = 0; q < n; ++q) dot += std::conj(basis[i][q]) * w[q];
                    h[j * (restart + 1) + i] += dot;
                    for (size_t q = 0; q < n; ++q) w[q] -= dot * basis[i][q];
                }
            double next = vnorm(w.data(), n);
            h[j * (restart + 1) + j + 1] = next;
            for (size_t i = 0; i < rot.size(); ++i) {
                int off = j * (restart + 1) + (int)i;
                cd a = h[off], b = h[off + 1];
                double c = rot[i].first;
                cd s = rot[i].second;
                h[off] = c * a + s * b;
                h[off + 1] = -std::conj(s) * a + c * b;
            }
            int dg = j * (restart + 1) + j;
            cd a = h[dg], b = h[dg + 1];
            double length = std::hypot(std::abs(a), std::abs(b));
            if (!std::isfinite(length) || length == 0.0) return 4;
            cd phase = std::abs(a) == 0.0 ? cd(1, 0) : a / std::abs(a);
            double c = std::abs(a) / length;
            cd s = phase * std::conj(b) / length;
            h[dg] = phase * length;
            h[dg + 1] = 0.0;
            rot.push_back({c, s});
            g[j + 1] = -std::conj(s) * g[j];
            g[j] *= c;
            used = j + 1;
            iterations += 1;
            if (std::abs(g[j + 1]) <= tol || next == 0.0 || iterations == max_iter) break;
            basis.emplace_back(n);
            for (size_t q = 0; q < n; ++q) basis.back()[q] = w[q] / next;
        }
        for (int i = used - 1; i >= 0; --i) {
            cd tail(0, 0);
            for (int jj = i + 1; jj < used; ++jj) tail += h[jj * (restart + 1) + i] * g[jj];
            g[i] = (g[i] - tail) / h[i * (restart + 1) + i];
            for (size_t q = 0; q < n; ++q) answer[q] += g[i] * basis[i][q];
        }
        apply(answer, prod.data());
        for (size_t q = 0; q < n; ++q) residual[q] = rhs[q] - prod[q];
    }
}

// =======================================================================================
// C interface for the tests (ctypes). Complex arrays are interleaved re, im doubles.
int ewald_table(int lmax, std::complex<double> k, const double* lattice, const double* kpar, const double* r,
                std::complex<double> eta, std::complex<double>* out);

extern "C" {

int orc_version() { return 1; }

double orc_wigner3j(int j1, int j2, int j3, int m1, int m2, int m3) { return wigner3j(j1, j2, j3, m1, m2, m3); }

// degrees of coupling.rs:146-160; returns count, writes up to cap values
int orc_degrees(int l, int m, int lambda, int mu, int cross, int* out, int cap) {
    std::vector<int> v;
    degrees(l, m, lambda, mu, cross != 0, v);
    for (int i = 0; i < (int)v.size() && i < cap; ++i) out[i] = v[i];
    return (int)v.size();
}

void orc_spherical_hankels(int last, double x, double* out) { spherical_hankels(last, x, (cd*)out); }
void orc_spherical_j(int last, double re, double im, double* out) { sph_j_sequence(last, cd(re, im), (cd*)out); }
void orc_spherical_h(int last, double re, double im, double* out) { sph_h_sequence(last, cd(re, im), (cd*)out); }

void orc_solid_table(int order, const double* unit, double* out) { solid_table(order, unit, (cd*)out); }

// number of plan terms for lmax (helicity plan)
int orc_plan_terms(int lmax) { return (int)plan_between(lmax, true).terms.size(); }

// M x M column-major block of the translation from source to destination at displacement
// pos = destination - source (sw/plan.rs:282-289); singular = outgoing Hankel radial
void orc_translation_block(int lmax, double k, const double* pos, int singular, int helicity, double* out) {
    Plan plan = plan_between(lmax, helicity != 0);
    plan_evaluate(plan, k, pos, singular != 0, (cd*)out);
}

// 2x2 Mie block of degree l in mode order, row-major
void orc_mie_block(int l, double size, double eps_re, double eps_im, double* out) {
    mie_block_mode_order(l, size, cd(eps_re, eps_im), (cd*)out);
}

// Cluster operator A = I - T C (cluster/spheres.rs:154-220, interaction.rs:158-169),
// column-major n x n, n = N * M. Also returns T blocks (N * lmax * 4 complex) if tb != null.
void orc_cluster_operator(int lmax, double k0, int N, const double* radii, const double* eps, const double* pos,
                          double* out, double* tb) {
    Plan plan = plan_between(lmax, true);
    int M = plan.M;
    size_t n = (size_t)N * M;
    cd* A = (cd*)out;
    std::vector<cd> T((size_t)N * lmax * 4);
    for (int i = 0; i < N; ++i)
        for (int l = 1; l <= lmax; ++l)
            mie_block_mode_order(l, k0 * radii[i], cd(eps[2 * i], eps[2 * i + 1]), &T[((size_t)i * lmax + l - 1) * 4]);
    if (tb) std::memcpy(tb, T.data(), T.size() * sizeof(cd));
    std::vector<Mode> md = modes(lmax);
    #pragma omp parallel
    {
        std::vector<cd> blk((size_t)M * M);
        #pragma omp for schedule(dynamic)
        for (int j = 0; j < N; ++j) {
            for (int i = 0; i < N; ++i) {
                if (i == j) {
                    for (int c = 0; c < M; ++c)
                        for (int r = 0; r < M; ++r)
                            A[((size_t)j * M + c) * n + (size_t)i * M + r] = (r == c) ? cd(1, 0) : cd(0, 0);
                    continue;
                }
                double d[3] = {pos[3 * i] - pos[3 * j], pos[3 * i + 1] - pos[3 * j + 1], pos[3 * i + 2] - pos[3 * j + 2]};
                plan_evaluate(plan, k0, d, true, blk.data());
                // -T_i C_ij : T_i acts on destination rows; 2x2 blocks on (l, m) row pairs
                for (int c = 0; c < M; ++c)
                    for (int r = 0; r < M; r += 2) {
                        int l = md[r].l;
                        const cd* t = &T[((size_t)i * lmax + l - 1) * 4];
                        cd c0 = blk[(size_t)c * M + r], c1 = blk[(size_t)c * M + r + 1];
                        A[((size_t)j * M + c) * n + (size_t)i * M + r] = -(t[0] * c0 + t[1] * c1);
                        A[((size_t)j * M + c) * n + (size_t)i * M + r + 1] = -(t[2] * c0 + t[3] * c1);
                    }
            }
        }
    }
}

// Incident plane waves (pw/expand.rs:308-360): B column c for wavevector kvec[c] (3 complex)
// with polarization pols[c], positions of N spheres; n x p column-major.
void orc_plane_wave_expansion(int lmax, int N, const double* pos, int p, const double* kvecs, const int* pols,
                              double* out) {
    std::vector<Mode> md = modes(lmax);
    int M = (int)md.size();
    size_t n = (size_t)N * M;
    cd* B = (cd*)out;
    for (int c = 0; c < p; ++c) {
        const cd* kv = (const cd*)(kvecs + 6 * c);
        std::vector<cd> ang(M);
        for (int e = 0; e < M; ++e) ang[e] = pw_to_sw(md[e], kv, pols[c]);
        for (int i = 0; i < N; ++i) {
            cd ph = pw_phase(kv, pos + 3 * i);
            for (int e = 0; e < M; ++e) B[c * n + (size_t)i * M + e] = ang[e] * ph;
        }
    }
}

// Dense solve (I - T C) X = T B with the restated LU. A is consumed (n x n), B is n x p;
// X = out. Returns 0 or a status code (3 = singular).
int orc_dense_solve(int lmax, int N, const double* Aop, const double* tb, const double* B, int p, double* X) {
    int M = 2 * lmax * (lmax + 2);
    int n = N * M;
    LuFactor f;
    f.n = n;
    f.a.assign((const cd*)Aop, (const cd*)Aop + (size_t)n * n);
    int st = lu_factor(f);
    if (st) return st;
    const cd* T = (const cd*)tb;
    cd* x = (cd*)X;
    const cd* b = (const cd*)B;
    std::vector<Mode> md = modes(lmax);
    for (int c = 0; c < p; ++c)
        for (int i = 0; i < N; ++i)
            for (int r = 0; r < M; r += 2) {
                const cd* t = &T[((size_t)i * lmax + md[r].l - 1) * 4];
                size_t o = (size_t)c * n + (size_t)i * M + r;
                x[o] = t[0] * b[o] + t[1] * b[o + 1];
                x[o + 1] = t[2] * b[o] + t[3] * b[o + 1];
            }
    lu_solve(f, x, p);
    return 0;
}

// Periodic array of one sphere per cell (cluster/interaction.rs:292-315 with
// sw/expansion.rs:418-454 and sw/plan.rs:383-413): S = evaluate_table(D_pm / N_pm) with the
// lattice sums at shift 0 (ewald.cpp), X = (I - T S)^-1 T, M x M column-major.
int orc_array_solve(int lmax, double k0, double radius, double eps_re, double eps_im, const double* lattice,
                    const double* kpar, double eta, double* out) {
    Plan plan = plan_between(lmax, true);
    int M = plan.M, order = plan.lmax;
    int T = (order + 1) * (order + 1);
    std::vector<cd> D(T), S((size_t)M * M);
    double r0[3] = {0.0, 0.0, 0.0};
    int st = ewald_table(order, cd(k0, 0.0), lattice, kpar, r0, cd(eta, 0.0), D.data());
    if (st) return st;
    for (int p = 0; p <= order; ++p)
        for (int m = -p; m <= p; ++m) {
            double nrm = std::sqrt((2 * p + 1) / (4 * M_PI)) * std::exp(0.5 * (log_factorial(p - m) - log_factorial(p + m)));
            D[p * p + p + m] /= nrm;
        }
    plan_evaluate_table(plan, D.data(), S.data());
    std::vector<Mode> md = modes(lmax);
    std::vector<cd> Tb((size_t)lmax * 4);
    for (int l = 1; l <= lmax; ++l) mie_block_mode_order(l, k0 * radius, cd(eps_re, eps_im), &Tb[(l - 1) * 4]);
    LuFactor f;
    f.n = M;
    f.a.assign((size_t)M * M, cd(0, 0));
    std::vector<cd> X((size_t)M * M, cd(0, 0));
    for (int c = 0; c < M; ++c)
        for (int r = 0; r < M; r += 2) {
            const cd* t = &Tb[(md[r].l - 1) * 4];
            cd s0 = S[(size_t)c * M + r], s1 = S[(size_t)c * M + r + 1];
            f.a[(size_t)c * M + r] = (r == c ? 1.0 : 0.0) - (t[0] * s0 + t[1] * s1);
            f.a[(size_t)c * M + r + 1] = (r + 1 == c ? 1.0 : 0.0) - (t[2] * s0 + t[3] * s1);
        }
    for (int c = 0; c < M; c += 2) {
        const cd* t = &Tb[(md[c].l - 1) * 4];
        X[(size_t)c * M + c] = t[0];
        X[(size_t)c * M + c + 1] = t[2];
        X[(size_t)(c + 1) * M + c] = t[1];
        X[(size_t)(c + 1) * M + c + 1] = t[3];
    }
    if ((st = lu_factor(f))) return st;
    lu_solve(f, X.data(), M);
    std::memcpy(out, X.data(), X.size() * sizeof(cd));
    return 0;
}

int orc_lu_solve(int n, const double* A, double* B, int p) {
    LuFactor f;
    f.n = n;
    f.a.assign((const cd*)A, (const cd*)A + (size_t)n * n);
    int st = lu_factor(f);
    if (st) return st;
    lu_solve(f, (cd*)B, p);
    return 0;
}

// Cross sections (python/treams_rs/_tmatrix.py:405-441) with flux 0.5 and factor 0.5:
// sca = Re(x^H O x) / k^2, ext = -Re(b^H x) / k^2, O the regular expansion between all
// positions (sw/expansion.rs:116-130). One column.
void orc_cross_sections(int lmax, double k0, int N, const double* pos, const double* x_, const double* b_,
                        double* sca, double* ext) {
    Plan plan = plan_between(lmax, true);
    int M = plan.M;
    size_t n = (size_t)N * M;
    const cd* x = (const cd*)x_;
    const cd* b = (const cd*)b_;
    double total = 0.0;
    #pragma omp parallel reduction(+ : total)
    {
        std::vector<cd> blk((size_t)M * M);
        #pragma omp for schedule(dynamic)
        for (int i = 0; i < N; ++i) {
            cd acc(0, 0);
            for (int j = 0; j < N; ++j) {
                double d[3] = {pos[3 * i] - pos[3 * j], pos[3 * i + 1] - pos[3 * j + 1], pos[3 * i + 2] - pos[3 * j + 2]};
                plan_evaluate(plan, k0, d, false, blk.data());
                for (int c = 0; c < M; ++c) {
                    cd xc = x[(size_t)j * M + c];
                    for (int r = 0; r < M; ++r) acc += std::conj(x[(size_t)i * M + r]) * blk[(size_t)c * M + r] * xc;
                }
            }
            total += acc.real();
        }
    }
    double e = 0.0;
    for (size_t q = 0; q < n; ++q) e += (std::conj(b[q]) * x[q]).real();
    *sca = total / (k0 * k0);
    *ext = -e / (k0 * k0);
}

// Matrix-free cluster (cluster/iterative.rs:99-284): y = (I - T C) x for p columns
void orc_iterative_apply(int lmax, double k0, int N, const double* radii, const double* eps, const double* pos,
                         const double* x_, int p, double* y_) {
    Plan plan = plan_between(lmax, true);
    int M = plan.M;
    size_t n = (size_t)N * M;
    std::vector<cd> T((size_t)N * lmax * 4);
    for (int i = 0; i < N; ++i)
        for (int l = 1; l <= lmax; ++l)
            mie_block_mode_order(l, k0 * radii[i], cd(eps[2 * i], eps[2 * i + 1]), &T[((size_t)i * lmax + l - 1) * 4]);
    std::vector<Mode> md = modes(lmax);
    const cd* x = (const cd*)x_;
    cd* y = (cd*)y_;
    #pragma omp parallel
    {
        std::vector<cd> blk((size_t)M * M), acc((size_t)M * p);
        #pragma omp for schedule(dynamic)
        for (int i = 0; i < N; ++i) {
            std::fill(acc.begin(), acc.end(), cd(0, 0));
            for (int j = 0; j < N; ++j) {
                if (j == i) continue;
                double d[3] = {pos[3 * i] - pos[3 * j], pos[3 * i + 1] - pos[3 * j + 1], pos[3 * i + 2] - pos[3 * j + 2]};
                plan_evaluate(plan, k0, d, true, blk.data());
                for (int c = 0; c < p; ++c)
                    for (int s = 0; s < M; ++s) {
                        cd xs = x[(size_t)c * n + (size_t)j * M + s];
                        for (int r = 0; r < M; ++r) acc[(size_t)c * M + r] += blk[(size_t)s * M + r] * xs;
                    }
            }
            for (int c = 0; c < p; ++c)
                for (int r = 0; r < M; r += 2) {
                    const cd* t = &T[((size_t)i * lmax + md[r].l - 1) * 4];
                    cd c0 = acc[(size_t)c * M + r], c1 = acc[(size_t)c * M + r + 1];
                    size_t o = (size_t)c * n + (size_t)i * M + r;
                    y[o] = x[o] - (t[0] * c0 + t[1] * c1);
                    y[o + 1] = x[o + 1] - (t[2] * c0 + t[3] * c1);
                }
        }
    }
}

// Matrix-free GMRES solve of (I - T C) X = T B (cluster/iterative.rs:236-284), one column
// at a time (the reference batches up to eight columns; batching changes no arithmetic).
int orc_iterative_solve(int lmax, double k0, int N, const double* radii, const double* eps, const double* pos,
                        const double* B, int p, double rtol, double atol, int restart, int max_iter, double* X,
                        int* iterations, double* residuals) {
    int M = 2 * lmax * (lmax + 2);
    size_t n = (size_t)N * M;
    std::vector<cd> T((size_t)N * lmax * 4);
    for (int i = 0; i < N; ++i)
        for (int l = 1; l <= lmax; ++l)
            mie_block_mode_order(l, k0 * radii[i], cd(eps[2 * i], eps[2 * i + 1]), &T[((size_t)i * lmax + l - 1) * 4]);
    std::vector<Mode> md = modes(lmax);
    const cd* b = (const cd*)B;
    int status = 0;
    for (int c = 0; c < p; ++c) {
        std::vector<cd> rhs(n);
        for (int i = 0; i < N; ++i)
            for (int r = 0; r < M; r += 2) {
                const cd* t = &T[((size_t)i * lmax + md[r].l - 1) * 4];
                size_t o = (size_t)i * M + r;
                rhs[o] = t[0] * b[c * n + o] + t[1] * b[c * n + o + 1];
                rhs[o + 1] = t[2] * b[c * n + o] + t[3] * b[c * n + o + 1];
            }
        auto apply = [&](const cd* xin, cd* yout) {
            orc_iterative_apply(lmax, k0, N, radii, eps, pos, (const double*)xin, 1, (double*)yout);
        };
        int st = gmres_solve(n, rhs.data(), (cd*)X + c * n, rtol, atol, restart, max_iter, apply, &iterations[c],
                             &residuals[c]);
        if (st) status = st;
    }
    return status;
}

// Generic GMRES on a dense matrix (tests of the GMRES restatement)
int orc_gmres_dense(int n, const double* A_, const double* b_, double rtol, int restart, int max_iter, double* x,
                    int* iterations, double* residual) {
    const cd* A = (const cd*)A_;
    auto apply = [&](const cd* xin, cd* yout) {
        for (int i = 0; i < n; ++i) yout[i] = 0.0;
        for (int j = 0; j < n; ++j)
            for (int i = 0; i < n; ++i) yout[i] += A[(size_t)j * n + i] * xin[j];
    };
    return gmres_solve(n, (const cd*)b_, (cd*)x, rtol, 0.0, restart, max_iter, apply, iterations, residual);
}

}  // extern "C"
