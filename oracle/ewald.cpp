// CPU oracle: test infrastructure only. Nothing in the product links or calls this file.
//
// 2D Ewald lattice sums of outgoing spherical waves and the special functions they take,
// restated from treams-core:
//   lattice/mod.rs:11-15      D_lm(k, kpar, r) = sum'_R h_l(k|r+R|) Y_lm(-r-R) e^{i kpar.R}
//   lattice/cell.rs:164-175   automatic split eta = sqrt(2 pi)/(k L) max(|k L|/8, 1)
//   lattice/ewald.rs:39-270, 610-665   real + reciprocal (+ self at r = 0), shift reduced
//                             into a cell with the Bloch phase e^{-i kpar.R0}
//   lattice/real.rs:149-187   real-space term -i sqrt(2/pi) k^l |rho|^l Y_lm I_2l(k|rho|, eta)
//   lattice/reciprocal.rs:288-334 (2D spherical summand), 22-60 (S_lmn), 467-487 (self term)
//   lattice/reduced.rs:18-100 F_n(v, 0) = Gamma(n, v)/(-v)^n on the outgoing sheet, and
//                             F_n(v, t) = sum_j (t/2)^j/j! F_(n-j)(v, 0) (reduced.rs:223)
//   lattice/sheets.rs          sheet of v per diffraction order, self sheet
//   special/integrals/kambe.rs:36-120  Kambe series I_n = eta^(n+1)/2 sum_j c^j/j! R((n+1)/2-j)
//   special/integrals/gamma.rs upper incomplete gamma Gamma(a, z)
// Everything runs in binary128 (__float128): where the reference keeps f64 accuracy with
// ladders, Kambe recurrences and rounding bounds, this restatement evaluates the plain
// series and continued fractions (DLMF 8.7.3, 8.4.15, 6.6.2, 8.9.2) with 34 digits, so
// their cancellation stays far below the 1e-13 the tables are checked to. Shells are
// added until the Gaussian factor of a shell is below e^-90 and two consecutive shells
// add less than 1e-26 of the part (the reference stops at 2e-13, shells.rs:34).
#include <quadmath.h>

#include <algorithm>
#include <cmath>
#include <complex>
#include <vector>

namespace {

typedef __float128 Q;

struct C {
    Q re, im;
};
inline C mk(Q r, Q i = 0) { return C{r, i}; }
inline C operator+(C a, C b) { return mk(a.re + b.re, a.im + b.im); }
inline C operator-(C a, C b) { return mk(a.re - b.re, a.im - b.im); }
inline C operator-(C a) { return mk(-a.re, -a.im); }
inline C operator*(C a, C b) { return mk(a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re); }
inline C operator*(Q s, C a) { return mk(s * a.re, s * a.im); }
inline C operator*(C a, Q s) { return mk(s * a.re, s * a.im); }
inline C operator/(C a, C b) {
    if (fabsq(b.re) >= fabsq(b.im)) {
        Q r = b.im / b.re, d = b.re + b.im * r;
        return mk((a.re + a.im * r) / d, (a.im - a.re * r) / d);
    }
    Q r = b.re / b.im, d = b.re * r + b.im;
    return mk((a.re * r + a.im) / d, (a.im * r - a.re) / d);
}
inline C operator/(C a, Q s) { return mk(a.re / s, a.im / s); }
inline C& operator+=(C& a, C b) { return a = a + b; }
inline C& operator*=(C& a, C b) { return a = a * b; }
inline Q cabs(C z) { return hypotq(z.re, z.im); }
// argument with the side of the negative real axis taken from the sign of a zero imaginary part
inline Q carg(C z) {
    if (z.im == 0) {
        if (z.re >= 0) return 0;
        return signbitq(z.im) ? -M_PIq : M_PIq;
    }
    return atan2q(z.im, z.re);
}
inline C cexp(C z) {
    Q e = expq(z.re);
    return mk(e * cosq(z.im), e * sinq(z.im));
}
inline C clog(C z) { return mk(logq(cabs(z)), carg(z)); }
inline C csqrt(C z) {  // principal root, lower side of the cut for a -0 imaginary part
    Q r = cabs(z);
    if (r == 0) return mk(0, 0);
    Q t = sqrtq(0.5Q * (r + fabsq(z.re)));
    if (z.re >= 0) return mk(t, z.im / (2 * t));
    return mk(fabsq(z.im) / (2 * t), copysignq(t, z.im));
}
inline C cpowr(C z, Q a) {  // principal z^a
    if (z.re == 0 && z.im == 0) return mk(0, 0);
    return cexp(a * clog(z));
}
inline C cpowi(C z, int n) {
    C r = mk(1, 0), b = z;
    unsigned e = (unsigned)(n < 0 ? -n : n);
    while (e) {
        if (e & 1) r = r * b;
        b = b * b;
        e >>= 1;
    }
    return n < 0 ? mk(1, 0) / r : r;
}
inline C lower_side(C z) {  // sheets.rs:12-17
    if (z.im == 0) z.im = -0.0Q;
    return z;
}
inline Q lfact(int n) { return lgammaq((Q)n + 1); }
inline std::complex<double> to_d(C z) { return {(double)z.re, (double)z.im}; }
inline C from_d(std::complex<double> z) { return mk(z.real(), z.imag()); }
const Q EULER = 0.5772156649015328606065120900824024310422Q;

// ---- upper incomplete gamma Gamma(a, z), principal branch (special/integrals/gamma.rs) --
bool is_nonpositive_integer(Q a) { return a <= 0 && a == floorq(a); }

// DLMF 8.7.3 / 8.4.15 / 6.6.2: power series about z = 0
C gamma_series(Q a, C z) {
    if (is_nonpositive_integer(a)) {
        int n = (int)(-a);
        // E1(z) = -gamma - ln z - sum_k (-z)^k / (k k!)
        C s = mk(0, 0), term = mk(1, 0);
        for (int k = 1; k < 4000; ++k) {
            term = term * (-z) / (Q)k;
            C add = term / (Q)k;
            s += add;
            if (cabs(add) <= 1e-40Q * cabs(s) && k > cabs(z)) break;
        }
        C e1 = mk(-EULER, 0) - clog(z) - s;
        if (n == 0) return e1;
        // Gamma(-n, z) = (-1)^n / n! (E1(z) - e^-z sum_{k<n} (-1)^k k! / z^(k+1))
        C fin = mk(0, 0), zp = mk(1, 0) / z;
        Q fk = 1;
        for (int k = 0; k < n; ++k) {
            if (k > 0) fk *= k;
            fin += ((k % 2) ? -fk : fk) * zp;
            zp = zp / z;
        }
        C g = e1 - cexp(-z) * fin;
        Q sign = (n % 2) ? -1 : 1;
        return (sign * expq(-lfact(n))) * g;
    }
    C s = mk(1 / a, 0), term = mk(1, 0);
    for (int k = 1; k < 4000; ++k) {
        term = term * (-z) / (Q)k;
        C add = term / (a + k);
        s += add;
        if (cabs(add) <= 1e-40Q * cabs(s) && k > cabs(z)) break;
    }
    return mk(tgammaq(a), 0) - cpowr(z, a) * s;
}

// DLMF 8.9.2 (even contraction of Legendre's continued fraction), modified Lentz
C gamma_fraction(Q a, C z) {
    const Q tiny = 1e-4000Q;
    C b = z + mk(1 - a, 0);
    C c = mk(1 / tiny, 0), d = mk(1, 0) / b, h = d;
    for (int i = 1; i < 20000; ++i) {
        Q an = -(Q)i * ((Q)i - a);
        b = b + mk(2, 0);
        d = an * d + b;
        if (cabs(d) < tiny) d = mk(tiny, 0);
        c = b + mk(an, 0) / c;
        if (cabs(c) < tiny) c = mk(tiny, 0);
        d = mk(1, 0) / d;
        C del = d * c;
        h = h * del;
        if (cabs(del - mk(1, 0)) < 1e-38Q) break;
    }
    return cexp(-z) * cpowr(z, a) * h;
}

C upper_gamma(Q a, C z) {
    if (a >= 1 && a <= 64 && a == floorq(a)) {
        // DLMF 8.4.8: Gamma(n, z) = (n-1)! e^-z sum_{k<n} z^k/k!, exact at its zeros
        int n = (int)a;
        C s = mk(0, 0), term = mk(1, 0);
        for (int k = 0; k < n; ++k) {
            if (k > 0) term = term * z / (Q)k;
            s += term;
        }
        return tgammaq(a) * (cexp(-z) * s);
    }
    Q az = cabs(z);
    bool fraction = (az >= 10 && z.re >= -0.6Q * az) || z.re >= 2;
    return fraction ? gamma_fraction(a, z) : gamma_series(a, z);
}

// ---- Kambe integrals I_n(z, eta) = int_eta^inf t^n exp(-z^2 t^2/2 + 1/(2 t^2)) dt --------
// special/integrals/kambe.rs:36-120: with a = (z eta)^2/2, c = 1/(2 eta^2) and
// R(d) = Gamma(d, a)/a^d, I_n = eta^(n+1)/2 sum_j c^j/j! R((n+1)/2 - j). Even orders take
// sqrt(a) = z eta/sqrt 2 with Re z >= 0; where that is minus the principal root (the
// reference's `reflected` ladder) R continues to R - 2 Gamma(d)/a^d (DLMF 8.2.10).
struct KambeLadder {
    C a;
    bool reflected = false;
    int parity = 0;  // 0: even orders (half-integer d), 1: odd orders (integer d)
    std::vector<C> cache;  // R at d = top/2 - i
    int top2 = 0;          // 2 d of cache[0]
    C at(int twice_d) {
        int i = (top2 - twice_d) / 2;
        while ((int)cache.size() <= i) {
            Q d = (Q)(top2 - 2 * (int)cache.size()) / 2;
            C ad = cpowr(a, d);
            C r = upper_gamma(d, a) / ad;
            if (reflected) r = r - mk(2 * tgammaq(d), 0) / ad;
            cache.push_back(r);
        }
        return cache[i];
    }
};

KambeLadder kambe_ladder(int top_order, C z, C eta) {
    KambeLadder L;
    L.parity = ((top_order % 2) + 2) % 2;
    if (L.parity == 0 && z.re < 0) z = -z;
    C ze = z * eta;
    L.a = 0.5Q * (ze * ze);
    if (L.parity == 0) {
        C root = csqrt(ze * ze);
        C conj_ze = mk(ze.re, -ze.im);
        L.reflected = (root * conj_ze).re < 0;
    }
    L.top2 = top_order + 1;
    return L;
}

C kambe_from(KambeLadder& L, int n, C eta) {
    C c = mk(0.5Q, 0) / (eta * eta);
    Q cn = cabs(c);
    C sum = mk(0, 0), coef = mk(1, 0);
    int last = (int)(200 + 3 * std::min((double)cn, 1000.0));
    for (int j = 0; j <= last; ++j) {
        if (j > 0) coef = coef * c / (Q)j;
        C term = coef * L.at(n + 1 - 2 * j);
        sum += term;
        if (j > 3 && j > cn && cabs(term) <= 1e-40Q * cabs(sum)) break;
    }
    return 0.5Q * cpowi(eta, n + 1) * sum;
}

C kambe(int n, C z, C eta) {
    KambeLadder L = kambe_ladder(n, z, eta);
    return kambe_from(L, n, eta);
}

// ---- solid harmonics |x|^l P_l^m(cos theta) e^{i m phi} (special/harmonics.rs:147-305) ----
void solid_table_q(int order, const Q x[3], std::vector<C>& table) {
    table.assign((size_t)(order + 1) * (order + 1), mk(0, 0));
    Q r2 = x[0] * x[0] + x[1] * x[1] + x[2] * x[2];
    C xy = mk(x[0], x[1]), diag = mk(1, 0);
    for (int o = 0; o <= order; ++o) {
        if (o > 0) diag = (-(Q)(2 * o - 1)) * (diag * xy);
        C p = diag, prev = mk(0, 0);
        for (int deg = o; deg <= order; ++deg) {
            if (deg > o) {
                Q a = (Q)(2 * deg - 1) / (Q)(deg - o), b = (Q)(deg + o - 1) / (Q)(deg - o);
                C next = (a * x[2]) * p - (b * r2) * prev;
                prev = p;
                p = next;
            }
            table[deg * deg + deg + o] = p;
            if (o > 0) {
                Q refl = ((o % 2) ? -1 : 1) * expq(lfact(deg - o) - lfact(deg + o));
                table[deg * deg + deg - o] = refl * mk(p.re, -p.im);
            }
        }
    }
}
Q harmonic_normalization(int l, int m) {  // harmonics.rs:139-141
    return sqrtq((Q)(2 * l + 1) / (4 * M_PIq)) * expq(0.5Q * (lfact(l - m) - lfact(l + m)));
}

// ---- sheets (lattice/sheets.rs) -------------------------------------------------------------
struct Split {
    C square;
    Q turn;
    bool has_near;
    Q near;
};
Split make_split(C k, C eta) {
    Split s;
    C ke = k * eta;
    s.square = k * k;
    s.turn = carg(ke * ke);
    Q angle = fabsq(s.turn) + 0.5Q;
    s.has_near = angle < M_PI_2q;
    s.near = s.has_near ? powq(tanq(angle), 2) : 0;
    return s;
}
// returns false for the principal sheet, else the argument of v on the sheet
bool split_sheet(const Split& s, C q2, Q& sheet) {
    C sq = s.square - q2;
    bool near = sq.re > 0 && sq.im * sq.im <= s.near * sq.re * sq.re;
    if (s.has_near && !near) return false;
    Q turn;
    if (sq.im == 0)
        turn = sq.re > 0 ? 0 : M_PIq;
    else {
        turn = carg(sq);
        if (turn < 0) turn += 2 * M_PIq;
    }
    sheet = turn - M_PIq - s.turn;
    return true;
}
Q sheet_turns(Q sheet, C value) { return roundq((sheet - carg(value)) / (2 * M_PIq)); }

// ---- reduced integrals F_n(v, t) (lattice/reduced.rs:18-100, 223-250) ------------------
C reduced_power(int twice_n, C z) {  // (-z)^n with the principal root for half-integer n
    int fl = (twice_n >= 0) ? twice_n / 2 : -((-twice_n + 1) / 2);
    C p = cpowi(-z, fl);
    if (twice_n % 2 != 0) p = p * csqrt(-z);
    return p;
}
// F_n(v, 0) on its sheet, `turns` whole turns from the principal argument (or none)
C gamma_limit(int twice_n, C value, bool has_turns, Q turns) {
    C z = lower_side(value);
    C rp = reduced_power(twice_n, z);
    C g = upper_gamma((Q)twice_n / 2, z) / rp;
    if (!has_turns) return g;
    if (twice_n % 2 != 0) {
        if (turns != 0 && fmodq(fabsq(turns), 2) == 1) g = g - mk(2 * tgammaq((Q)twice_n / 2), 0) / rp;
        if (z.im > 0) g = -g;
    } else if (twice_n <= 0 && turns != 0) {
        int n = -twice_n / 2;
        g = g - mk(0, 2 * M_PIq * turns) * cpowi(value, n) * expq(-lfact(n));
    }
    return g;
}

// ---- one Ewald evaluation: every (l, m) up to lmax ---------------------------------------
struct Lattice2 {
    Q a[2][2], b[2][2], area;
};
Lattice2 make_lattice(const double* rows) {
    Lattice2 L;
    for (int i = 0; i < 2; ++i)
        for (int j = 0; j < 2; ++j) L.a[i][j] = rows[2 * i + j];
    Q det = L.a[0][0] * L.a[1][1] - L.a[0][1] * L.a[1][0];
    L.area = fabsq(det);
    // b_i . a_j = 2 pi delta_ij
    L.b[0][0] = 2 * M_PIq * L.a[1][1] / det;
    L.b[0][1] = -2 * M_PIq * L.a[1][0] / det;
    L.b[1][0] = -2 * M_PIq * L.a[0][1] / det;
    L.b[1][1] = 2 * M_PIq * L.a[0][0] / det;
    return L;
}

enum { PART_REAL = 1, PART_RECIPROCAL = 2 };

// status: 0 ok, 1 invalid input, 4 not converged
int ewald_table_q(int lmin, int lmax, C k, const double* rows, const double* kpar_d, const double* r_d, C eta,
                  int parts, std::vector<C>& out) {
    const int T = (lmax + 1) * (lmax + 1);
    out.assign(T, mk(0, 0));
    if (!(k.im >= 0) || !(k.re >= 0) || (k.re == 0 && k.im == 0) || lmax < 0 || lmax > 24) return 1;
    Lattice2 L = make_lattice(rows);
    if (!(L.area > 0)) return 1;
    if (eta.re == 0 && eta.im == 0) {  // cell.rs:164-175
        C e = mk(1, 0) / (k * mk(sqrtq(L.area), 0));
        Q scale = std::max(0.125Q / cabs(e), (Q)1);
        eta = (sqrtq(2 * M_PIq) * scale) * e;
    }
    Q kpar[2] = {kpar_d[0], kpar_d[1]};
    // reduce the shift into a cell (ewald.rs:610-665): r' = r - R0, phase e^{-i kpar.R0}
    Q r[3] = {r_d[0], r_d[1], r_d[2]};
    Q frac0 = (L.b[0][0] * r[0] + L.b[0][1] * r[1]) / (2 * M_PIq);
    Q frac1 = (L.b[1][0] * r[0] + L.b[1][1] * r[1]) / (2 * M_PIq);
    Q c0 = roundq(frac0), c1 = roundq(frac1);
    Q R0[2] = {c0 * L.a[0][0] + c1 * L.a[1][0], c0 * L.a[0][1] + c1 * L.a[1][1]};
    r[0] -= R0[0];
    r[1] -= R0[1];
    C cell_phase = cexp(mk(0, -(kpar[0] * R0[0] + kpar[1] * R0[1])));
    const bool at_origin = r[0] == 0 && r[1] == 0 && r[2] == 0;

    std::vector<C> real(T, mk(0, 0)), recip(T, mk(0, 0));
    std::vector<Q> norm(T);
    for (int l = 0; l <= lmax; ++l)
        for (int m = -l; m <= l; ++m) norm[l * l + l + m] = harmonic_normalization(l, m);
    C ke = k * eta;
    const Q len1 = hypotq(L.a[0][0], L.a[0][1]), len2 = hypotq(L.a[1][0], L.a[1][1]);
    const Q hdir = L.area / std::max(len1, len2);
    const Q blen1 = hypotq(L.b[0][0], L.b[0][1]), blen2 = hypotq(L.b[1][0], L.b[1][1]);
    const Q hrec = (4 * M_PIq * M_PIq / L.area) / std::max(blen1, blen2);
    const Q rin = hypotq(r[0], r[1]), kpn = hypotq(kpar[0], kpar[1]);
    const int max_shells = 400;

    auto shell_points = [](int s, std::vector<std::pair<int, int>>& pts) {
        pts.clear();
        if (s == 0) {
            pts.push_back({0, 0});
            return;
        }
        for (int i = -s; i <= s; ++i) {
            pts.push_back({i, -s});
            pts.push_back({i, s});
        }
        for (int j = -s + 1; j <= s - 1; ++j) {
            pts.push_back({-s, j});
            pts.push_back({s, j});
        }
    };
    auto shell_max = [&](const std::vector<C>& add) {
        Q mx = 0;
        for (auto& v : add) mx = std::max(mx, cabs(v));
        return mx;
    };
    auto part_scale = [&](const std::vector<C>& s) {
        Q mx = 1;
        for (auto& v : s) mx = std::max(mx, cabs(v));
        return mx;
    };
    std::vector<std::pair<int, int>> pts;

    if (parts & PART_REAL) {
        // real.rs:149-187 at rho = -r - R, Bloch factor e^{i kpar.R}
        Q decay = (ke * ke).re;
        if (!(decay > 0)) return 4;
        int floor_s = (int)ceilq((sqrtq(2 * 40 / decay) + rin) / hdir) + 1;
        int quiet = 0;
        std::vector<C> add(T);
        for (int s = 0; s < max_shells; ++s) {
            std::fill(add.begin(), add.end(), mk(0, 0));
            shell_points(s, pts);
            std::vector<std::vector<C>> per(pts.size());
#pragma omp parallel for schedule(dynamic)
            for (size_t pi = 0; pi < pts.size(); ++pi) {
                const auto& nn = pts[pi];
                std::vector<C>& acc = per[pi];
                acc.assign(T, mk(0, 0));
                Q R[2] = {nn.first * L.a[0][0] + nn.second * L.a[1][0], nn.first * L.a[0][1] + nn.second * L.a[1][1]};
                Q rho[3] = {-r[0] - R[0], -r[1] - R[1], -r[2]};
                Q dist = sqrtq(rho[0] * rho[0] + rho[1] * rho[1] + rho[2] * rho[2]);
                if (dist == 0) continue;
                std::vector<C> tab;
                solid_table_q(lmax, rho, tab);
                C z = k * mk(dist, 0);
                KambeLadder lad = kambe_ladder(2 * lmax, z, eta);
                C bloch = cexp(mk(0, kpar[0] * R[0] + kpar[1] * R[1]));
                C kl = cpowi(k, lmin);
                for (int l = lmin; l <= lmax; ++l) {
                    if (l > lmin) kl = kl * k;
                    C radial = kambe_from(lad, 2 * l, eta);
                    C f = mk(0, -sqrtq(2 / M_PIq)) * kl * radial * bloch;
                    for (int m = -l; m <= l; ++m) acc[l * l + l + m] += (norm[l * l + l + m] * tab[l * l + l + m]) * f;
                }
            }
            for (auto& acc : per)  // fixed order: results do not depend on the thread count
                for (int i = 0; i < T; ++i) add[i] += acc[i];
            for (int i = 0; i < T; ++i) real[i] += add[i];
            Q mx = shell_max(add);
            quiet = (mx <= 1e-26Q * part_scale(real)) ? quiet + 1 : 0;
            if (s >= floor_s && quiet >= 2) break;
            if (s == max_shells - 1) return 4;
        }
    }
    if (parts & PART_RECIPROCAL) {
        // reciprocal.rs:288-334 with the phase e^{-i q.r}; sheets per order (sheets.rs)
        C inv = mk(1, 0) / (ke * ke);
        Q decay = inv.re;
        if (!(decay > 0)) return 4;
        int floor_s = (int)ceilq((sqrtq(2 * 60 / decay) + kpn) / hrec) + 1;
        Split split = make_split(k, eta);
        const bool use_sheet = k.im >= 0 && (k * eta).re > 0;
        C zz = k * mk(r[2], 0);
        C t = (zz * eta) * (zz * eta);
        const bool on_plane = r[2] == 0;
        // terms of the t-series: (t/2)^j / j! until below 1e-40 of the largest
        int J = 0;
        if (!on_plane) {
            Q tn = cabs(t) / 2, term = 1, big = 1;
            for (J = 1; J < 400; ++J) {
                term *= tn / J;
                big = std::max(big, term);
                if (J > tn && term < 1e-40Q * big) break;
            }
        }
        Q sq2 = sqrtq((Q)2);
        std::vector<C> pref(T);
        for (int l = 0; l <= lmax; ++l)
            for (int m = -l; m <= l; ++m) {
                // sqrt(2l+1) (-i)^m sqrt((l+m)!(l-m)!) / (A k^2 (-2)^l)
                C mi = cpowi(mk(0, -1), m);
                Q mag = sqrtq((Q)(2 * l + 1)) * expq(0.5Q * (lfact(l + m) + lfact(l - m))) /
                        (L.area * powq(-2, l));
                pref[l * l + l + m] = mag * mi / (k * k);
            }
        int quiet = 0;
        std::vector<C> add(T);
        for (int s = 0; s < max_shells; ++s) {
            std::fill(add.begin(), add.end(), mk(0, 0));
            shell_points(s, pts);
            std::vector<std::vector<C>> per(pts.size());
            int failed = 0;
#pragma omp parallel for schedule(dynamic)
            for (size_t pi = 0; pi < pts.size(); ++pi) {
                const auto& nn = pts[pi];
                std::vector<C>& acc = per[pi];
                acc.assign(T, mk(0, 0));
                std::vector<C> limits, F(lmax + 1);
                Q q[2] = {kpar[0] + nn.first * L.b[0][0] + nn.second * L.b[1][0],
                          kpar[1] + nn.first * L.b[0][1] + nn.second * L.b[1][1]};
                C q2 = mk(q[0] * q[0] + q[1] * q[1], 0);
                C beta2 = q2 / (k * k);
                C v = (beta2 - mk(1, 0)) / (2.0Q * (eta * eta));
                v = lower_side(v);
                if (cabs(v) <= 1e-14Q) {  // reciprocal.rs:236-241: on a diffraction threshold
#pragma omp atomic write
                    failed = 1;
                    continue;
                }
                bool has_turns = false;
                Q turns = 0;
                if (use_sheet) {
                    Q sheet;
                    has_turns = true;
                    if (split_sheet(split, q2, sheet)) turns = sheet_turns(sheet, lower_side(v));
                }
                // limits F_(1/2 - i)(v, 0), i = 0..lmax + J
                limits.resize(lmax + J + 1);
                for (int i = 0; i <= lmax + J; ++i) limits[i] = gamma_limit(1 - 2 * i, v, has_turns, turns);
                for (int n = 0; n <= lmax; ++n) {
                    if (on_plane) {
                        F[n] = limits[n];
                        continue;
                    }
                    C acc = mk(0, 0), w = mk(1, 0);
                    for (int j = 0; j <= J; ++j) {
                        if (j > 0) w = w * t / (Q)(2 * j);
                        acc += w * limits[n + j];
                    }
                    F[n] = acc;
                }
                C phase = cexp(mk(0, -(q[0] * r[0] + q[1] * r[1])));
                for (int l = lmin; l <= lmax; ++l)
                    for (int m = -l; m <= l; ++m) {
                        int am = m < 0 ? -m : m;
                        C az = mk(q[0], m < 0 ? -q[1] : q[1]) / k;
                        C azp = cpowi(az, am);
                        C sum = mk(0, 0);
                        C factor = mk(1, 0) / (sq2 * eta);
                        for (int n = 0; n <= l - am; ++n) {
                            // S_lmn (reciprocal.rs:22-60)
                            C poly = mk(0, 0);
                            for (int sidx = n; sidx <= std::min(l - am, 2 * n); ++sidx) {
                                if ((l - am - sidx) % 2 != 0) continue;
                                int zp = 2 * n - sidx;
                                if (on_plane && zp > 0) continue;
                                C zterm = cpowi(-zz, zp);
                                Q lw = -lfact(2 * n - sidx) - lfact(sidx - n) - lfact((l + am - sidx) / 2) -
                                       lfact((l - am - sidx) / 2);
                                poly += zterm * cpowi(beta2, (l - sidx - am) / 2) * expq(lw);
                            }
                            if (poly.re != 0 || poly.im != 0) sum += factor * F[n] * poly;
                            factor = factor * (2.0Q * (eta * eta));
                        }
                        acc[l * l + l + m] += pref[l * l + l + m] * sum * azp * phase;
                    }
            }
            if (failed) return 1;
            for (auto& acc : per)
                for (int i = 0; i < T; ++i) add[i] += acc[i];
            for (int i = 0; i < T; ++i) recip[i] += add[i];
            Q mx = shell_max(add);
            quiet = (mx <= 1e-26Q * part_scale(recip)) ? quiet + 1 : 0;
            if (s >= floor_s && quiet >= 2) break;
            if (s == max_shells - 1) return 4;
        }
        if (at_origin) {
            // self term (reciprocal.rs:467-487): only l = 0 survives at r = 0
            C value = lower_side(mk(-0.5Q, 0) / (eta * eta));
            C kk = k;
            if (kk.im == 0) kk.im = 0;
            C ka = 0.5Q * (k * k) * (eta * eta);
            Q self_sheet = 2 * carg(kk) - M_PIq - carg(ka);
            Q turns = sheet_turns(self_sheet, value);
            C g = upper_gamma(-0.5Q, value);
            if (fmodq(fabsq(turns), 2) == 1) g = mk(2 * tgammaq(-0.5Q), 0) - g;
            recip[0] += (norm[0] * (0.5Q / sqrtq(M_PIq))) * g;
        }
    }
    for (int i = 0; i < T; ++i) out[i] = cell_phase * (real[i] + recip[i]);
    return 0;
}

}  // namespace

// C++ entry for the periodic-array oracle in oracle.cpp: D_lm for every l <= lmax
int ewald_table(int lmax, std::complex<double> k, const double* lattice, const double* kpar, const double* r,
                std::complex<double> eta, std::complex<double>* out) {
    std::vector<C> v;
    int st = ewald_table_q(0, lmax, from_d(k), lattice, kpar, r, from_d(eta), PART_REAL | PART_RECIPROCAL, v);
    for (size_t i = 0; i < v.size(); ++i) out[i] = to_d(v[i]);
    return st;
}

extern "C" {

// Gamma(a, z); a zero imaginary part selects the side of the cut by its sign
int orc_upper_gamma(double a, double zre, double zim, double* out) {
    C g = upper_gamma((Q)a, mk(zre, zim));
    out[0] = (double)g.re;
    out[1] = (double)g.im;
    return 0;
}

int orc_kambe(int n, double zre, double zim, double eta_re, double eta_im, double* out) {
    C v = kambe(n, mk(zre, zim), mk(eta_re, eta_im));
    out[0] = (double)v.re;
    out[1] = (double)v.im;
    return 0;
}

// one D_lm; part 0 full, 1 real space, 2 reciprocal (with the self term)
int orc_lsumsw2d(int l, int m, double kre, double kim, const double* lattice, const double* kpar, const double* r,
                 double eta_re, double eta_im, int part, double* out) {
    if (l < 0 || m < -l || m > l) return 1;
    int parts = part == 1 ? PART_REAL : part == 2 ? PART_RECIPROCAL : (PART_REAL | PART_RECIPROCAL);
    std::vector<C> v;
    int st = ewald_table_q(l, l, mk(kre, kim), lattice, kpar, r, mk(eta_re, eta_im), parts, v);
    out[0] = (double)v[l * l + l + m].re;
    out[1] = (double)v[l * l + l + m].im;
    return st;
}

// every D_lm, l <= lmax, table index l*l+l+m
int orc_lsumsw2d_table(int lmax, double kre, double kim, const double* lattice, const double* kpar, const double* r,
                       double eta_re, double eta_im, double* out) {
    std::vector<C> v;
    int st = ewald_table_q(0, lmax, mk(kre, kim), lattice, kpar, r, mk(eta_re, eta_im), PART_REAL | PART_RECIPROCAL, v);
    for (size_t i = 0; i < v.size(); ++i) {
        out[2 * i] = (double)v[i].re;
        out[2 * i + 1] = (double)v[i].im;
    }
    return st;
}

}  // extern "C"
