// Row and column equilibration of the assembled operator before its LU factorization
// (linalg/mod.rs:137-228 of treams-core: equilibrate only when the entries spread, then
// row scales r_i = 1/max_j |a_ij| and column scales c_j = 1/max_i r_i |a_ij|, xGEEQU-style,
// with |z| = max(|Re z|, |Im z|)). Here every scale is rounded to a power of two, so scaling
// is exact in FP64 and FP32 storage. The factorization then holds A' = R A C and a solve
// computes x = C A'^-1 (R b).
//
// Kernels: row maxima over column chunks (threads over rows, coalesced column reads, one
// partial per (row, chunk)) reduced in a fixed order; column maxima of R A (a warp per four
// columns of the magnitude mirror below); one in-place scaling pass (threads over rows, column
// chunks). HBM-bound.
//
// Then the balancing sweeps of linalg/mod.rs:229-310 (Sinkhorn and Knopp: unit magnitude sums
// determine the scaled operator, whatever the units): every column factor y_j, then every row
// factor x_i, moves by the power of two that puts its scaled magnitude sum into
// [ln 2, 2 ln 2); sweeps stop after one that moves no factor by more than 2 (at most 64). A sum
// that is not normal leaves the max scales alone; so do factors beyond 2^+-256. Two passes over
// the matrix per sweep: column sums (CTA per column) and row sums (threads over rows, partial
// per column chunk, fixed-order reduction). The column maxima and the sweeps read a bfloat16
// mirror of |a_ij| (written by the row-maxima pass) with the max scales applied on the fly, and A
// is scaled once at the end: three passes over A plus (1 + 2 sweeps) over the 2-byte mirror.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <vector>

#include "common.cuh"
#include "kernels.h"

namespace tcu {

namespace {

constexpr int EQ_CHUNKS = 32;
// bfloat16 magnitude mirror at the end of the scratch, 256-byte aligned
inline size_t mirror_offset(int n) { return ((size_t)(EQ_CHUNKS + 4) * n + (n + 255) / 256 + 1 + 31) / 32 * 32; }
inline size_t mirror_doubles(int n) { return ((size_t)n * n * 2 + 255) / 256 * 32; }

template <typename C>
__device__ __forceinline__ double mag(C v) {
    return fmax(fabs((double)v.x), fabs((double)v.y));
}
// Magnitude mirror: the column and balancing passes read |a_ij| as bfloat16 (8-bit mantissa,
// the FP32 exponent range), a quarter of the complex64 bytes and an eighth of complex128. The
// scales are powers of two chosen from magnitude sums; a sum off by < 0.5 % moves a choice only
// when the sum sits at a boundary, and the scaling stays exact either way.
__device__ __forceinline__ uint16_t to_bf16(double m) {
    const unsigned b = __float_as_uint((float)m);
    if ((b & 0x7f800000u) == 0x7f800000u) return (uint16_t)(b >> 16);  // inf, NaN
    return (uint16_t)((b + 0x7fffu + ((b >> 16) & 1u)) >> 16);       // round to nearest even
}
__device__ __forceinline__ double mag(uint16_t v) { return (double)__uint_as_float((unsigned)v << 16); }

// row maxima, and the bfloat16 magnitude mirror M (column-major like A)
template <typename C>
__global__ void row_max_partial(const C* __restrict__ A, int n, double* __restrict__ partial,
                                uint16_t* __restrict__ mirror) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int chunk = blockIdx.y;
    if (i >= n) return;
    const int per = (n + EQ_CHUNKS - 1) / EQ_CHUNKS;
    const int j0 = chunk * per, j1 = min(n, j0 + per);
    double m = 0.0;
    for (int j = j0; j < j1; ++j) {
        const double v = mag(A[(size_t)j * n + i]);
        mirror[(size_t)j * n + i] = to_bf16(v);
        m = fmax(m, v);
    }
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

// a thread per row over a chunk of columns (the grid of row_max_partial): r_i stays in a
// register, c_j is a broadcast load, and the column loop keeps several loads in flight
template <typename C>
__global__ void apply_scales(C* __restrict__ A, int n, const double* __restrict__ r, const double* __restrict__ c) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int per = (n + EQ_CHUNKS - 1) / EQ_CHUNKS;
    const int j0 = blockIdx.y * per, j1 = min(n, j0 + per);
    const double ri = r[i];
#pragma unroll 4
    for (int j = j0; j < j1; ++j) {
        const double s = ri * c[j];
        C v = A[(size_t)j * n + i];
        v.x = (decltype(v.x))((double)v.x * s);
        v.y = (decltype(v.y))((double)v.y * s);
        A[(size_t)j * n + i] = v;
    }
}

__global__ void scale_rows_kernel(cplx* __restrict__ v, const double* __restrict__ s, size_t n, int ncol) {
    const size_t total = n * (size_t)ncol;
    for (size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x; t < total; t += (size_t)gridDim.x * blockDim.x)
        v[t] = cscale(v[t], s[t % n]);
}

// Column maxima of R A on the mirror (n even): a warp per BAL_COLS columns, two rows per 4-byte
// word, the row scales loaded once for all of the warp's columns; fixed-order warp reduction.
constexpr int BAL_COLS = 4;
__device__ __forceinline__ double lo16(uint32_t v) { return (double)__uint_as_float(v << 16); }
__device__ __forceinline__ double hi16(uint32_t v) { return (double)__uint_as_float(v & 0xffff0000u); }

__global__ void col_scale_mirror(const uint16_t* __restrict__ Mg, int n, const double* __restrict__ r,
                                 double* __restrict__ c) {
    const int lane = threadIdx.x & 31;
    const int j0 = (blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5)) * BAL_COLS;
    if (j0 >= n) return;
    const uint32_t* col[BAL_COLS];
    double m[BAL_COLS];
#pragma unroll
    for (int t = 0; t < BAL_COLS; ++t) {
        col[t] = reinterpret_cast<const uint32_t*>(Mg + (size_t)min(j0 + t, n - 1) * n);
        m[t] = 0.0;
    }
    for (int q = lane; q < n / 2; q += 32) {
        const double r0 = r[2 * q], r1 = r[2 * q + 1];
#pragma unroll
        for (int t = 0; t < BAL_COLS; ++t) {
            const uint32_t v = col[t][q];
            m[t] = fmax(m[t], fmax(r0 * lo16(v), r1 * hi16(v)));
        }
    }
#pragma unroll
    for (int t = 0; t < BAL_COLS; ++t) {
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) m[t] = fmax(m[t], __shfl_xor_sync(0xffffffffu, m[t], off));
        if (lane == 0 && j0 + t < n) c[j0 + t] = m[t] > 0.0 ? exp2(-rint(log2(m[t]))) : 1.0;
    }
}

// ---- balancing sweeps ---------------------------------------------------------------------
constexpr int BAL_SWEEPS = 64;
enum : int { BAL_COARSE = 1, BAL_ABORT = 2, BAL_UNFIT = 4 };

// factor *= 1 / (largest power of two <= sum * factor / ln 2); flags the step's size
__device__ __forceinline__ void bal_advance(double& factor, double sum, int* flags) {
    const double ratio = sum * factor / 0.69314718055994530942;
    const unsigned long long bits = (unsigned long long)__double_as_longlong(ratio);
    const unsigned long long ex = bits & 0x7ff0000000000000ULL;
    if (ex == 0 || ex == 0x7ff0000000000000ULL || ratio < 0.0) {  // zero, subnormal, inf, NaN
        atomicOr(flags, BAL_ABORT);
        return;
    }
    const double step = 1.0 / __longlong_as_double((long long)ex);
    factor *= step;
    if (step < 0.5 || step > 2.0) atomicOr(flags, BAL_COARSE);
}

// The sweeps run on R A C without forming it: |a_ij| r_i c_j with the max scales r, c, read
// from the bfloat16 mirror M two rows (one 4-byte word; n is even) at a time. Row weights
// w_i = x_i r_i and column weights cy_j = c_j y_j are kept beside the factors.

// column sums: a warp per BAL_COLS columns (the row weights loaded once for all of them),
// fixed-order warp reduction per column
__global__ void bal_col_kernel(const uint16_t* __restrict__ Mg, int n, const double* __restrict__ w,
                               const double* __restrict__ c, double* __restrict__ y, double* __restrict__ cy,
                               int* flags) {
    const int lane = threadIdx.x & 31;
    const int j0 = (blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5)) * BAL_COLS;
    if (j0 >= n) return;
    const uint32_t* col[BAL_COLS];
    double s[BAL_COLS];
#pragma unroll
    for (int t = 0; t < BAL_COLS; ++t) {
        col[t] = reinterpret_cast<const uint32_t*>(Mg + (size_t)min(j0 + t, n - 1) * n);
        s[t] = 0.0;
    }
    for (int q = lane; q < n / 2; q += 32) {
        const double w0 = w[2 * q], w1 = w[2 * q + 1];
#pragma unroll
        for (int t = 0; t < BAL_COLS; ++t) {
            const uint32_t v = col[t][q];
            s[t] = fma(w0, lo16(v), s[t]);
            s[t] = fma(w1, hi16(v), s[t]);
        }
    }
#pragma unroll
    for (int t = 0; t < BAL_COLS; ++t) {
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) s[t] += __shfl_xor_sync(0xffffffffu, s[t], off);
        const int j = j0 + t;
        if (lane == 0 && j < n) {
            double yy = y[j];
            bal_advance(yy, s[t] * c[j], flags);
            y[j] = yy;
            cy[j] = c[j] * yy;
        }
    }
}

// row sums over a chunk of columns: a thread per pair of rows, 4-byte loads coalesced over the warp
__global__ void bal_row_partial(const uint16_t* __restrict__ Mg, int n, const double* __restrict__ cy,
                                double* __restrict__ partial) {
    const int i2 = blockIdx.x * blockDim.x + threadIdx.x;
    if (2 * i2 >= n) return;
    const int per = (n + EQ_CHUNKS - 1) / EQ_CHUNKS;
    const int j0 = blockIdx.y * per, j1 = min(n, j0 + per);
    double s0 = 0.0, s1 = 0.0;
#pragma unroll 8
    for (int j = j0; j < j1; ++j) {
        const uint32_t v = reinterpret_cast<const uint32_t*>(Mg + (size_t)j * n)[i2];
        const double wj = cy[j];
        s0 = fma(lo16(v), wj, s0);
        s1 = fma(hi16(v), wj, s1);
    }
    partial[(size_t)blockIdx.y * n + 2 * i2] = s0;
    partial[(size_t)blockIdx.y * n + 2 * i2 + 1] = s1;
}

__global__ void bal_row_update(const double* __restrict__ partial, int n, const double* __restrict__ r,
                               double* __restrict__ x, double* __restrict__ w, int* flags) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double s = 0.0;
    for (int c = 0; c < EQ_CHUNKS; ++c) s += partial[(size_t)c * n + i];
    double xx = x[i];
    bal_advance(xx, s * r[i], flags);
    x[i] = xx;
    w[i] = xx * r[i];
}

// x = y = 1, w = r, cy = c
__global__ void bal_init_kernel(int n, const double* __restrict__ r, const double* __restrict__ c,
                                double* __restrict__ x, double* __restrict__ y, double* __restrict__ w,
                                double* __restrict__ cy) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    x[i] = 1.0;
    y[i] = 1.0;
    w[i] = r[i];
    cy[i] = c[i];
}

// factors within 2^+-256 and normal products with the max scales, else BAL_UNFIT
__global__ void bal_fit_kernel(int n, const double* __restrict__ x, const double* __restrict__ y,
                               const double* __restrict__ r, const double* __restrict__ c, int* flags) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double lo = 8.636168555094445e-78, hi = 1.157920892373162e77;  // 2^-256, 2^256
    const double a = x[i], b = y[i], ra = r[i] * a, cb = c[i] * b;
    const bool ok = a >= lo && a <= hi && b >= lo && b <= hi && isfinite(ra) && isfinite(cb) &&
                    fabs(ra) >= 2.2250738585072014e-308 && fabs(cb) >= 2.2250738585072014e-308;
    if (!ok) atomicOr(flags, BAL_UNFIT);
}

__global__ void bal_fold_kernel(int n, const double* __restrict__ x, const double* __restrict__ y, double* __restrict__ r,
                                double* __restrict__ c) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    r[i] *= x[i];
    c[i] *= y[i];
}


// Balancing sweeps over R A C (A unscaled, mirror Mg of |A|, max scales r and c); on success r
// and c take the factors (the caller then scales A once). scratch: x, y, w, cy (n each),
// partial (EQ_CHUNKS n), flags.
tcu_status balance_impl(const uint16_t* Mg, int n, double* r, double* c, double* scratch, int* sweeps_out,
                        cudaStream_t st, long long* launches) {
    double* x = scratch;
    double* y = x + n;
    double* w = y + n;
    double* cy = w + n;
    double* partial = cy + n;
    int* d_flags = reinterpret_cast<int*>(partial + (size_t)EQ_CHUNKS * n);
    const int nb = (n + 255) / 256, nb2 = (n / 2 + 255) / 256;
    bal_init_kernel<<<nb, 256, 0, st>>>(n, r, c, x, y, w, cy);
    if (launches) ++*launches;
    int flags = 0, sweep = 0;
    for (; sweep < BAL_SWEEPS; ++sweep) {
        if (cudaMemsetAsync(d_flags, 0, sizeof(int), st) != cudaSuccess) return TCU_DEVICE_ERROR;
        bal_col_kernel<<<(n + 8 * BAL_COLS - 1) / (8 * BAL_COLS), 256, 0, st>>>(Mg, n, w, c, y, cy, d_flags);
        bal_row_partial<<<dim3(nb2, EQ_CHUNKS), 256, 0, st>>>(Mg, n, cy, partial);
        bal_row_update<<<nb, 256, 0, st>>>(partial, n, r, x, w, d_flags);
        if (launches) *launches += 3;
        if (cudaMemcpyAsync(&flags, d_flags, sizeof(int), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
            cudaStreamSynchronize(st) != cudaSuccess)
            return TCU_DEVICE_ERROR;
        if (flags & BAL_ABORT) {  // a sum that is not normal: keep the max scales
            *sweeps_out = -(sweep + 1);
            return TCU_OK;
        }
        if (!(flags & BAL_COARSE)) break;
    }
    if (cudaMemsetAsync(d_flags, 0, sizeof(int), st) != cudaSuccess) return TCU_DEVICE_ERROR;
    bal_fit_kernel<<<nb, 256, 0, st>>>(n, x, y, r, c, d_flags);
    if (launches) ++*launches;
    if (cudaMemcpyAsync(&flags, d_flags, sizeof(int), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess)
        return TCU_DEVICE_ERROR;
    if (flags & BAL_UNFIT) {
        *sweeps_out = -(sweep + 1);
        return TCU_OK;
    }
    bal_fold_kernel<<<nb, 256, 0, st>>>(n, x, y, r, c);
    if (launches) *launches += 1;
    *sweeps_out = std::min(sweep + 1, BAL_SWEEPS);
    return TCU_OK;
}

template <typename C>
tcu_status equilibrate_impl(C* A, int n, double threshold, double* r, double* c, double* partial, bool* applied,
                            cudaStream_t st, long long* launches) {
    *applied = false;
    const int nb = (n + 255) / 256;
    uint16_t* mirror = reinterpret_cast<uint16_t*>(partial + mirror_offset(n));
    row_max_partial<C><<<dim3(nb, EQ_CHUNKS), 256, 0, st>>>(A, n, partial, mirror);
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
    if (n % 2 == 0)
        col_scale_mirror<<<(n + 8 * BAL_COLS - 1) / (8 * BAL_COLS), 256, 0, st>>>(mirror, n, r, c);
    else
        col_scale<uint16_t><<<n, 256, 0, st>>>(mirror, n, r, c);
    if (launches) ++*launches;
    int sweeps = 0;
    const tcu_status s = (n % 2 == 0) ? balance_impl(mirror, n, r, c, partial, &sweeps, st, launches) : TCU_OK;
    if (s) return s;
    apply_scales<C><<<dim3(nb, EQ_CHUNKS), 256, 0, st>>>(A, n, r, c);  // R A C with the balanced (or max) scales
    if (launches) ++*launches;
    *applied = true;
    return TCU_OK;
}

}  // namespace

size_t equilibrate_scratch_doubles(int n) { return mirror_offset(n) + mirror_doubles(n); }

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
