// Per-pair device helpers shared by the pair kernels and the preconditioners: the harmonic
// table of one sphere pair (one warp), the plan's term sums and the degree of an lm index.
#pragma once
#include "common.cuh"
#include "plan.h"

namespace tcu {

constexpr int MAXP = 22;  // radial orders p <= 2 lmax <= 20 (+1)

// ---- per-pair harmonic table ------------------------------------------------------------
// One warp fills Z (tsize complex) for displacement d = r_dest - r_src. Lanes 0..order each
// compute one order column. singular: outgoing Hankel radial; else regular j_p.
__device__ __forceinline__ void pair_table(const DevPlan& P, double k, double dx, double dy, double dz, bool singular,
                                           cplx* Z, int lane) {
    double r, u[3];
    bool ok = unit_direction(dx, dy, dz, r, u);
    if (!ok) {
        for (int t = lane; t < P.tsize; t += 32) Z[t] = mk(0.0, 0.0);
        if (lane == 0 && !singular) Z[0] = mk(1.0, 0.0);
        return;
    }
    if (lane > P.order) return;
    cplx rad[MAXP];
    if (singular) {
        hankel_sequence<MAXP>(P.order, k * r, rad);
    } else {
        double j[MAXP];
        bessel_j_sequence<MAXP>(P.order, k * r, j);
        for (int q = 0; q <= P.order && q < MAXP; ++q) rad[q] = mk(j[q], 0.0);
    }
    int m = lane;
    cplx xy = mk(u[0], u[1]);
    double z = u[2], r2 = u[0] * u[0] + u[1] * u[1] + u[2] * u[2];
    cplx diag = mk(1.0, 0.0);
    for (int q = 1; q <= m; ++q) diag = cscale(cmul(diag, xy), -double(2 * q - 1));
    cplx p = diag, prev = mk(0.0, 0.0);
    for (int deg = m; deg <= P.order; ++deg) {
        if (deg > m) {
            double a = double(2 * deg - 1) / double(deg - m);
            double b = double(deg + m - 1) / double(deg - m);
            cplx next = mk(a * z * p.x - b * r2 * prev.x, a * z * p.y - b * r2 * prev.y);
            prev = p;
            p = next;
        }
        Z[deg * deg + deg + m] = cmul(rad[deg], p);
        if (m > 0) {
            int idx = deg * deg + deg - m;
            Z[idx] = cmul(rad[deg], cscale(cconj(p), P.reflection[idx]));
        }
    }
}

// A and B term sums of combo c against table Z
__device__ __forceinline__ void combo_sums(const DevPlan& P, int c, const cplx* Z, cplx& A, cplx& B) {
    plan_combo_sums(P, c, Z, A, B);
}

__device__ __forceinline__ int degree_of(int lm) {  // lm = l*l - 1 + l + m
    int l = (int)sqrt((double)(lm + 1));
    while (l * l > lm + 1) --l;
    while ((l + 1) * (l + 1) <= lm + 1) ++l;
    return l;
}

}  // namespace tcu
