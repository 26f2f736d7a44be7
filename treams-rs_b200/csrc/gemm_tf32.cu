// Trailing update of the mixed-precision LU on the tcgen05 tensor cores (placeholder).
#include <cuda_runtime.h>

#include "kernels.h"
#include "precond.h"

namespace tcu {

bool tf32_enabled() { return false; }

void launch_tf32_update(float2*, int, int, int, LuWork&, cudaStream_t, long long*) {}

}  // namespace tcu
