// Translation plan shared by the host builder (plan.cpp) and the device kernels.
#pragma once
#include <vector_types.h>

#include <cstdint>
#include <vector>

namespace tcu {

// Host copy: combo[2c] = first term, combo[2c+1] = nA | nB << 16 for c = s * nlm + d
// (source (l,m) index s, destination index d, lm index = l*l - 1 + l + m); terms are the
// A list then the B list; idx = table index p*p+p+m-mu, w = interleaved complex weight.
struct HostPlan {
    int L = 0, nlm = 0, order = 0;
    std::vector<int> combo;
    std::vector<uint16_t> idx;
    std::vector<double> w;
    std::vector<double> reflection;  // (order+1)^2 negative-order factors, table order
};

HostPlan build_plan(int L);
double wigner3j_racah(int j1, int j2, int j3, int m1, int m2, int m3);

// Device view of a plan (pointers into device memory).
struct DevPlan {
    int L, nlm, order, tsize;  // tsize = (order + 1)^2
    const int2* combo;
    const uint16_t* idx;
    const double2* w;
    const double* reflection;
};

#ifdef __CUDACC__
// A (same-helicity) and B (cross) term sums of combo c = s * nlm + d against a harmonic table Z
__device__ __forceinline__ void plan_combo_sums(const DevPlan& P, int c, const double2* Z, double2& A, double2& B) {
    int2 cb = __ldg(&P.combo[c]);
    int t = cb.x, na = cb.y & 0xffff, nb = cb.y >> 16;
    A = make_double2(0.0, 0.0);
    B = make_double2(0.0, 0.0);
    for (int e = 0; e < na; ++e, ++t) {
        double2 w = __ldg(&P.w[t]), z = Z[__ldg(&P.idx[t])];
        A.x = fma(w.x, z.x, fma(-w.y, z.y, A.x));
        A.y = fma(w.x, z.y, fma(w.y, z.x, A.y));
    }
    for (int e = 0; e < nb; ++e, ++t) {
        double2 w = __ldg(&P.w[t]), z = Z[__ldg(&P.idx[t])];
        B.x = fma(w.x, z.x, fma(-w.y, z.y, B.x));
        B.y = fma(w.x, z.y, fma(w.y, z.x, B.y));
    }
}
#endif

}  // namespace tcu
