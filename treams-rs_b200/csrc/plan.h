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
    std::vector<uint8_t> idx;
    std::vector<double> w;
    std::vector<double> reflection;  // (order+1)^2 negative-order factors, table order
};

HostPlan build_plan(int L);
double wigner3j_racah(int j1, int j2, int j3, int m1, int m2, int m3);

// Device view of a plan (pointers into device memory).
struct DevPlan {
    int L, nlm, order, tsize;  // tsize = (order + 1)^2
    const int2* combo;
    const uint8_t* idx;
    const double2* w;
    const double* reflection;
};

}  // namespace tcu
