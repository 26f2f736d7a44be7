// Row and column equilibration of the assembled operator before its LU factorization
// (linalg/mod.rs:137-228 of treams-core: equilibrate only when the entries spread, then
// row scales r_i = 1/max_j |a_ij| and column scales c_j = 1/max_i r_i |a_ij|, xGEEQU-style,
// with |z| = max(|Re z|, |Im z|)). Here every scale is rounded to a power of two, so scaling
// is exact in FP64 and FP32 storage. The factorization then holds A' = R A C and a solve
// computes x = C A'^-1 (R b).
//
// Kernels: row maxima over column chunks (threads over rows, coalesced column reads, one
// partial per (row, chunk)) reduced in a fixed order; column maxima of R A (CTA per column);
// one in-place scaling pass. Three passes over the matrix: HBM-bound.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <vector>

#include "common.cuh"
#include "kernels.h"

namespace tcu {

namespace {

constexpr int EQ_CHUNKS = 32;

template <typename C>
__device__ __forceinline__ double mag(C v) {
    return fmax(fabs((double)v.x), fabs((double)v.y));
}

template <typename C>
__global__ void row_max_partial(const C* __restrict__ A, int n, double* __restrict__ partial) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int chunk = blockIdx.y;
    if (i >= n) return;
    const int per = (n + EQ_CHUNKS - 1) / EQ_CHUNKS;
    const int j0 = chunk * per, j1 = min(n, j0 + per);
    double m = 0.0;
    for (int j = j0; j < j1; ++j) m = fmax(m, mag(A[(size_t)j * n + i]));
    partial[(size_t)chunk * n + i] = m;
}

// r_i = 2^-round(log2 max_i), 1 for an all-zero row; also the global maximum (per block)
__global__ void row_scale(const double* __restrict__ partial, int n, double* __restrict__ r,
                          double* __restrict__ block_max) {
    __shared__ double sh[256];
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    double m = 0.0;
    if (i < n) {
        for (int c = 0; c < EQ_CHUNKS; ++c) m = fmax(m, partial[(size_t)c * n + i]);
        r[i] = m > 0.0 ? exp2(-rint(log2(m))) : 1.0;
    }
    sh[threadIdx.x] = m;
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s) sh[threadIdx.x] = fmax(sh[threadIdx.x], sh[threadIdx.x + s]);
        __syncthreads();
    }
    if (threadIdx.x == 0) block_max[blockIdx.x] = sh[0];
}

template <typename C>
__global__ void col_scale(const C* __restrict__ A, int n, const double* __restrict__ r, double* __restrict__ c) {
    __shared__ double sh[256];
    const int j = blockIdx.x;
    double m = 0.0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) m = fmax(m, r[i] * mag(A[(size_t)j * n + i]));
    sh[threadIdx.x] = m;
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s) sh[threadIdx.x] = fmax(sh[threadIdx.x], sh[threadIdx.x + s]);
        __syncthreads();
    }
    if (threadIdx.x == 0) c[j] = sh[0] > 0.0 ? exp2(-rint(log2(sh[0]))) : 1.0;
}

template <typename C>
__global__ void apply_scales(C* __restrict__ A, int n, const double* __restrict__ r, const double* __restrict__ c) {
    const size_t total = (size_t)n * n;
    for (size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x; t < total; t += (size_t)gridDim.x * blockDim.x) {
        const int i = (int)(t % n), j = (int)(t / n);
        const double s = r[i] * c[j];
        C v = A[t];
        v.x = (decltype(v.x))((double)v.x * s);
        v.y = (decltype(v.y))((double)v.y * s);
        A[t] = v;
    }
}

__global__ void scale_rows_kernel(cplx* __restrict__ v, const double* __restrict__ s, size_t n, int ncol) {
    const size_t total = n * (size_t)ncol;
    for (size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x; t < total; t += (size_t)gridDim.x * blockDim.x)
        v[t] = cscale(v[t], s[t % n]);
}

template <typename C>
tcu_status equilibrate_impl(C* A, int n, double threshold, double* r, double* c, double* partial, bool* applied,
                            cudaStream_t st, long long* launches) {
    *applied = false;
    const int nb = (n + 255) / 256;
    row_max_partial<C><<<dim3(nb, EQ_CHUNKS), 256, 0, st>>>(A, n, partial);
    double* block_max = partial + (size_t)EQ_CHUNKS * n;
    row_scale<<<nb, 256, 0, st>>>(partial, n, r, block_max);
    if (launches) *launches += 2;
    std::vector<double> bm(nb);
    if (cudaMemcpyAsync(bm.data(), block_max, nb * sizeof(double), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess)
        return TCU_DEVICE_ERROR;
    double mx = 0.0;
    for (double v : bm) mx = std::max(mx, v);
    if (!(mx > threshold)) return TCU_OK;  // entries within the spread a unit diagonal tolerates
    col_scale<C><<<n, 256, 0, st>>>(A, n, r, c);
    apply_scales<C><<<148 * 16, 256, 0, st>>>(A, n, r, c);
    if (launches) *launches += 2;
    *applied = true;
    return TCU_OK;
}

}  // namespace

size_t equilibrate_scratch_doubles(int n) { return (size_t)EQ_CHUNKS * n + (n + 255) / 256; }

tcu_status equilibrate(void* A, bool fp32, int n, double threshold, double* r, double* c, double* partial,
                       bool* applied, cudaStream_t st, long long* launches) {
    StageScope sc(ST_ASSEMBLE, st);
    if (fp32) return equilibrate_impl((float2*)A, n, threshold, r, c, partial, applied, st, launches);
    return equilibrate_impl((double2*)A, n, threshold, r, c, partial, applied, st, launches);
}

void scale_rows(cplx* v, const double* s, size_t n, int ncol, cudaStream_t st) {
    scale_rows_kernel<<<148 * 4, 256, 0, st>>>(v, s, n, ncol);
}

}  // namespace tcu
