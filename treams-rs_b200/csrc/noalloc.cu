// Allocation-free variant of the matrix-free cluster operator y = (I - T C) x.
//
// Some callers cannot allocate device memory: code running inside another framework's
// memory budget, or a host program that must not touch the CUDA allocator while a
// capture or a fixed memory plan is active. tcu_cluster_apply_noalloc takes device
// pointers for every input and output and keeps its scratch (the translation plan of the
// requested lmax, the Mie T blocks and a status word) in one file-scope device array of
// NOALLOC_BYTES. The array exists on every GPU that loads this library, for the life of
// the process. Host code only ever sees a host-side stand-in for its name, so its device
// address is looked up once per device (cudaGetSymbolAddress, with that device current)
// on the first call on that device. Every call copies the plan from pageable host memory
// and synchronises its stream to read the geometry check and the status word, so it cannot
// run inside a stream capture. Every call overwrites the whole used part of the array (the
// status word is cleared at the start), and calls that overlap on the GPU, on any streams,
// race on it.
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <mutex>

#include "../../include/treams_cuda.h"
#include "kernels.h"
#include "plan.h"

namespace tcu {

void set_error_message(const char* msg);

constexpr size_t NOALLOC_BYTES = (size_t)8 << 20;  // 8 MiB
static __device__ __align__(256) unsigned char g_noalloc_scratch[NOALLOC_BYTES];

namespace {

struct NoallocDevice {
    bool ready = false;
    unsigned char* base = nullptr;  // device address of g_noalloc_scratch
};
std::mutex g_noalloc_mu;
NoallocDevice g_noalloc_dev[64];
HostPlan g_noalloc_plans[8];  // host plan tables per lmax (1..7), built on first use
bool g_noalloc_plan_ready[8] = {};

tcu_status noalloc_fail(tcu_status s, const char* msg) {
    set_error_message(msg);  // read back with tcu_last_error_message()
    return s;
}

size_t up256(size_t v) { return (v + 255) & ~(size_t)255; }

// Geometry checks of cluster/spheres.rs:99-133 on the device: positive finite radii,
// finite permittivities and positions, no touching or overlapping pair.
__global__ void validate_kernel(int N, const double* __restrict__ radii, const double2* __restrict__ eps,
                                const double* __restrict__ pos, int* __restrict__ status) {
    long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    long long pairs = (long long)N * N;
    if (t >= pairs) return;
    int i = (int)(t / N), j = (int)(t % N);
    if (i == j) {
        double r = radii[i];
        double2 e = eps[i];
        if (!(isfinite(r) && r > 0.0) || !isfinite(e.x) || !isfinite(e.y) || !isfinite(pos[3 * i]) ||
            !isfinite(pos[3 * i + 1]) || !isfinite(pos[3 * i + 2]))
            atomicExch(status, 1);
        return;
    }
    if (j > i) return;
    double d = hypot(hypot(pos[3 * i] - pos[3 * j], pos[3 * i + 1] - pos[3 * j + 1]), pos[3 * i + 2] - pos[3 * j + 2]);
    if (!(d > radii[i] + radii[j]) || !isfinite(d)) atomicExch(status, 1);
}

}  // namespace

size_t noalloc_capacity() { return NOALLOC_BYTES; }

}  // namespace tcu

using namespace tcu;

extern "C" tcu_status tcu_cluster_apply_noalloc(void* stream, int lmax, double k0, size_t N, const double* radii,
                                                const double* eps, const double* positions, int p, const double* x,
                                                double* y) {
    if (lmax < 1 || lmax > 7 || !std::isfinite(k0) || k0 <= 0.0 || N == 0 || p <= 0 || !radii || !eps ||
        !positions || !x || !y)
        return noalloc_fail(TCU_INVALID_INPUT,
                            "require 1 <= lmax <= 7, positive finite k0, N >= 1, p >= 1 and device pointers");
    cudaStream_t st = (cudaStream_t)stream;
    cudaGetLastError();  // an earlier failure of the caller's own work is not this call's
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64)
        return noalloc_fail(TCU_DEVICE_ERROR, "no current CUDA device");
    std::lock_guard<std::mutex> lock(g_noalloc_mu);
    NoallocDevice& D = g_noalloc_dev[dev];
    if (!D.ready) {
        void* ptr = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&ptr, g_noalloc_scratch);
        if (e != cudaSuccess || !ptr) return noalloc_fail(TCU_DEVICE_ERROR, "cudaGetSymbolAddress of the scratch failed");
        D.base = (unsigned char*)ptr;
        pairs_init_attributes();
        D.ready = true;
    }
    if (!g_noalloc_plan_ready[lmax]) {
        g_noalloc_plans[lmax] = build_plan(lmax);
        g_noalloc_plan_ready[lmax] = true;
    }
    const HostPlan& h = g_noalloc_plans[lmax];
    const size_t ncombo = (size_t)h.nlm * h.nlm, nterm = h.idx.size();
    // scratch layout: status | combo | weights | reflection | term indices | T blocks
    size_t o_status = 0, o_combo = 256, o_w = up256(o_combo + ncombo * 8), o_refl = up256(o_w + nterm * 16),
           o_idx = up256(o_refl + h.reflection.size() * 8), o_t = up256(o_idx + nterm * 2);
    size_t need = o_t + N * (size_t)lmax * 4 * sizeof(double2);  // o_t follows the 2-byte term indices
    if (need > NOALLOC_BYTES)
        return noalloc_fail(TCU_INVALID_INPUT,
                            "cluster too large for the 8 MiB allocation-free scratch (N * lmax * 64 bytes plus the "
                            "translation plan must fit); use tcu_cluster_apply");
    unsigned char* b = D.base;
    int* status = (int*)(b + o_status);
    double2* T = (double2*)(b + o_t);
    const size_t M = 2 * (size_t)lmax * (lmax + 2), n = N * M;
    auto ck = [&](cudaError_t e) { return e == cudaSuccess; };
    if (!ck(cudaMemsetAsync(status, 0, sizeof(int), st)) ||
        !ck(cudaMemcpyAsync(b + o_combo, h.combo.data(), ncombo * 8, cudaMemcpyHostToDevice, st)) ||
        !ck(cudaMemcpyAsync(b + o_w, h.w.data(), nterm * 16, cudaMemcpyHostToDevice, st)) ||
        !ck(cudaMemcpyAsync(b + o_refl, h.reflection.data(), h.reflection.size() * 8, cudaMemcpyHostToDevice, st)) ||
        !ck(cudaMemcpyAsync(b + o_idx, h.idx.data(), nterm * 2, cudaMemcpyHostToDevice, st)))
        return noalloc_fail(TCU_DEVICE_ERROR, "copy of the translation plan into the scratch failed");
    long long pairs = (long long)N * N;
    validate_kernel<<<(unsigned)((pairs + 255) / 256), 256, 0, st>>>((int)N, radii, (const double2*)eps, positions,
                                                                     status);
    int hst = 0;
    if (!ck(cudaGetLastError()) || !ck(cudaMemcpyAsync(&hst, status, sizeof(int), cudaMemcpyDeviceToHost, st)) ||
        !ck(cudaStreamSynchronize(st)))
        return noalloc_fail(TCU_DEVICE_ERROR, "geometry check failed to run");
    if (hst)
        return noalloc_fail(TCU_INVALID_INPUT,
                            "require positive finite radii, finite permittivities and positions, and spheres that "
                            "neither touch nor overlap");
    launch_mie(lmax, k0, (int)N, radii, (const double2*)eps, T, status, st);
    if (!ck(cudaGetLastError())) return noalloc_fail(TCU_DEVICE_ERROR, "Mie coefficients failed to launch");
    DevPlan P;
    P.L = lmax;
    P.nlm = h.nlm;
    P.order = h.order;
    P.tsize = (h.order + 1) * (h.order + 1);
    P.combo = (const int2*)(b + o_combo);
    P.w = (const double2*)(b + o_w);
    P.reflection = (const double*)(b + o_refl);
    P.idx = (const uint16_t*)(b + o_idx);
    for (int c0 = 0; c0 < p; c0 += 8) {
        int nc = p - c0 < 8 ? p - c0 : 8;
        launch_apply(P, (int)N, k0, positions, T, (const double2*)x + (size_t)c0 * n, n, nc, nullptr, 1.0, -1.0, true,
                     (double2*)y + (size_t)c0 * n, st);
    }
    if (!ck(cudaGetLastError()) || !ck(cudaMemcpyAsync(&hst, status, sizeof(int), cudaMemcpyDeviceToHost, st)) ||
        !ck(cudaStreamSynchronize(st)) || !ck(cudaGetLastError()))
        return noalloc_fail(TCU_DEVICE_ERROR, "matrix-free operator failed to run");
    // the status words of the context path: 5 singular, 8 a bounded wait gave up, else a device fault
    if (hst == 5) return noalloc_fail(TCU_SINGULAR, "Mie coefficients: numerically singular");
    if (hst == 8) return noalloc_fail(TCU_TIMEOUT, "matrix-free operator: a device-side wait gave up");
    if (hst != 0) return noalloc_fail(TCU_DEVICE_ERROR, "matrix-free operator: nonzero device status");
    return TCU_OK;
}
