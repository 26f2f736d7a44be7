// Vector kernels on FP64 complex columns with fixed-order two-stage reductions, so that
// norms and dot products repeat bit for bit from run to run (the reference's results do
// not depend on its thread count, numerics/parallel.rs).
#include <cuda_runtime.h>

#include "common.cuh"
#include "kernels.h"

namespace tcu {

constexpr int RG = 256;  // partial sums per reduction (grid size of stage 1)

__device__ __forceinline__ double block_sum(double v, double* sh) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) sh[warp] = v;
    __syncthreads();
    double s = 0.0;
    if (threadIdx.x == 0)
        for (int q = 0; q < (int)(blockDim.x >> 5); ++q) s += sh[q];
    __syncthreads();
    return s;  // valid in thread 0
}

// stage 1: partial[c * RG + b] = sum over the fixed slice of column c of f(i)
__global__ void norm_stage1(const cplx* __restrict__ x, size_t n, double* __restrict__ partial) {
    __shared__ double sh[32];
    int c = blockIdx.y, b = blockIdx.x;
    const cplx* xc = x + (size_t)c * n;
    double s = 0.0;
    for (size_t i = (size_t)b * blockDim.x + threadIdx.x; i < n; i += (size_t)RG * blockDim.x) s += cabs2(xc[i]);
    s = block_sum(s, sh);
    if (threadIdx.x == 0) partial[c * RG + b] = s;
}
__global__ void sum_stage2(const double* __restrict__ partial, int ncol, double* __restrict__ out, int do_sqrt) {
    __shared__ double sh[32];
    int c = blockIdx.x;
    double s = partial[c * RG + threadIdx.x];
    s = block_sum(s, sh);
    if (threadIdx.x == 0) out[c] = do_sqrt ? sqrt(s) : s;
}
void vec_norms(const cplx* x, size_t n, int ncol, double* out_dev, double* partial, cudaStream_t st) {
    norm_stage1<<<dim3(RG, ncol), 256, 0, st>>>(x, n, partial);
    sum_stage2<<<ncol, RG, 0, st>>>(partial, ncol, out_dev, 1);
}

__global__ void rdot_stage1(const cplx* __restrict__ a, const cplx* __restrict__ b, size_t n, double* __restrict__ partial) {
    __shared__ double sh[32];
    int c = blockIdx.y, bl = blockIdx.x;
    const cplx* ac = a + (size_t)c * n;
    const cplx* bc = b + (size_t)c * n;
    double s = 0.0;
    for (size_t i = (size_t)bl * blockDim.x + threadIdx.x; i < n; i += (size_t)RG * blockDim.x)
        s += ac[i].x * bc[i].x + ac[i].y * bc[i].y;
    s = block_sum(s, sh);
    if (threadIdx.x == 0) partial[c * RG + bl] = s;
}
void vec_real_dots(const cplx* a, const cplx* b, size_t n, int ncol, double* out_dev, double* partial,
                   cudaStream_t st) {
    rdot_stage1<<<dim3(RG, ncol), 256, 0, st>>>(a, b, n, partial);
    sum_stage2<<<ncol, RG, 0, st>>>(partial, ncol, out_dev, 0);
}

// complex dots out[i] = sum conj(V_i) w, i < nv
__global__ void dots_stage1(const cplx* __restrict__ V, size_t ldv, const cplx* __restrict__ w, size_t n,
                            cplx* __restrict__ partial) {
    __shared__ double sh[32];
    int i = blockIdx.y, b = blockIdx.x;
    const cplx* v = V + (size_t)i * ldv;
    double sr = 0.0, si = 0.0;
    for (size_t q = (size_t)b * blockDim.x + threadIdx.x; q < n; q += (size_t)RG * blockDim.x) {
        cplx a = v[q], c = w[q];
        sr += a.x * c.x + a.y * c.y;
        si += a.x * c.y - a.y * c.x;
    }
    sr = block_sum(sr, sh);
    si = block_sum(si, sh);
    if (threadIdx.x == 0) partial[i * RG + b] = mk(sr, si);
}
__global__ void dots_stage2(const cplx* __restrict__ partial, cplx* __restrict__ out) {
    __shared__ double sh[32];
    int i = blockIdx.x;
    cplx p = partial[i * RG + threadIdx.x];
    double r = block_sum(p.x, sh);
    double im = block_sum(p.y, sh);
    if (threadIdx.x == 0) out[i] = mk(r, im);
}
void vec_dots(const cplx* V, size_t ldv, int nv, const cplx* w, size_t n, cplx* out_dev, cplx* partial,
              cudaStream_t st) {
    dots_stage1<<<dim3(RG, nv), 256, 0, st>>>(V, ldv, w, n, partial);
    dots_stage2<<<nv, RG, 0, st>>>(partial, out_dev);
}

__global__ void gemv_sub_kernel(cplx* __restrict__ w, const cplx* __restrict__ V, size_t ldv, int nv,
                                const cplx* __restrict__ h, size_t n) {
    size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= n) return;
    cplx acc = w[q];
    for (int i = 0; i < nv; ++i) {
        cplx hv = h[i], v = V[(size_t)i * ldv + q];
        acc.x -= hv.x * v.x - hv.y * v.y;
        acc.y -= hv.x * v.y + hv.y * v.x;
    }
    w[q] = acc;
}
void vec_gemv_sub(cplx* w, const cplx* V, size_t ldv, int nv, const cplx* h_dev, size_t n, cudaStream_t st) {
    gemv_sub_kernel<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(w, V, ldv, nv, h_dev, n);
}
__global__ void lincomb_kernel(cplx* __restrict__ x, const cplx* __restrict__ V, size_t ldv, int nv,
                               const cplx* __restrict__ g, size_t n) {
    size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= n) return;
    cplx acc = x[q];
    for (int i = nv - 1; i >= 0; --i) cfma(acc, g[i], V[(size_t)i * ldv + q]);
    x[q] = acc;
}
void vec_lincomb(cplx* x, const cplx* V, size_t ldv, int nv, const cplx* g_dev, size_t n, cudaStream_t st) {
    lincomb_kernel<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(x, V, ldv, nv, g_dev, n);
}
__global__ void axpy_kernel(cplx* __restrict__ y, const cplx* __restrict__ x, size_t total) {
    size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (q < total) y[q] = cadd(y[q], x[q]);
}
void vec_axpy(cplx* y, const cplx* x, size_t n, int ncol, cudaStream_t st) {
    size_t t = n * ncol;
    axpy_kernel<<<(unsigned)((t + 255) / 256), 256, 0, st>>>(y, x, t);
}
__global__ void sub_kernel(cplx* o, const cplx* a, const cplx* b, size_t total) {  // o may alias a or b
    size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (q < total) o[q] = csub(a[q], b[q]);
}
void vec_sub(cplx* out, const cplx* a, const cplx* b, size_t n, int ncol, cudaStream_t st) {
    size_t t = n * ncol;
    sub_kernel<<<(unsigned)((t + 255) / 256), 256, 0, st>>>(out, a, b, t);
}
__global__ void scale_kernel(cplx* o, const cplx* x, size_t n, double s) {  // o may alias x
    size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (q < n) o[q] = cscale(x[q], s);
}
void vec_scale_copy(cplx* out, const cplx* x, size_t n, double s, cudaStream_t st) {
    scale_kernel<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(out, x, n, s);
}

}  // namespace tcu
