// 2D Ewald lattice sums and the batched periodic-array solve (placeholder).
#include "../../include/treams_cuda.h"

extern "C" tcu_status tcu_lsumsw2d_batch(tcu_context*, int, double, const double*, size_t, const double*, double,
                                         double*) {
    return TCU_INVALID_INPUT;
}
extern "C" tcu_status tcu_array_solve_batch(tcu_context*, int, double, double, const double*, const double*, size_t,
                                            const double*, double, double*) {
    return TCU_INVALID_INPUT;
}
