// Block-Jacobi preconditioner of the matrix-free GMRES on A = I - T C (new here: the
// reference's iterative solver, cluster/iterative.rs:264-284 with linalg/gmres.rs:119, runs
// unpreconditioned). Spheres are grouped into blocks of up to 96 modes (3 spheres at lmax 3,
// 2 at lmax 4, 1 from lmax 5 on, where it is the identity since (I - T C)_ii = I): each sphere
// in Morton order that is still free opens a block and takes its nearest free neighbours. Every
// block's own system is inverted exactly (one CTA per block: assembly, pivoted LU and inverse
// in shared memory). The two-level preconditioners are in gnn.cu.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <numeric>
#include <vector>

#include "kernels.h"
#include "pairtable.cuh"
#include "precond.h"
#include "smem_lu.cuh"
#include "nearfield.cuh"

namespace tcu {

namespace {

using namespace nearfield;

constexpr int PB_MAXMODES = 96;  // modes per block (shared-memory LU)
constexpr int PB_PANEL = 48;

// Inverse of every block's system (I - T C)_bb; CTA per block, dinv stride PB_MAXMODES^2.
__global__ void __launch_bounds__(512) blk_inverse_kernel(DevPlan P, double k, const double* __restrict__ pos,
                                                          const cplx* __restrict__ T, const int* __restrict__ bptr,
                                                          const int* __restrict__ bmem, cplx* __restrict__ dinv,
                                                          int* __restrict__ status) {
    extern __shared__ double2 bi_smem[];
    __shared__ int piv[PB_MAXMODES];
    __shared__ int sing;
    const int b = blockIdx.x, M = 2 * P.nlm;
    const int m0 = bptr[b], cnt = bptr[b + 1] - m0, nb = cnt * M;
    double2* A = bi_smem;         // nb x nb
    double2* Bp = A + nb * nb;    // nb x PB_PANEL, the harmonic table aliases it
    const int tid = threadIdx.x, nth = blockDim.x;
    for (int t = tid; t < nb * nb; t += nth) A[t] = mk((t % nb) == (t / nb) ? 1.0 : 0.0, 0.0);
    __syncthreads();
    for (int a = 0; a < cnt; ++a)
        for (int c = 0; c < cnt; ++c) {
            if (a == c) continue;
            const int i = bmem[m0 + a], j = bmem[m0 + c];
            if (tid < 32)
                pair_table(P, k, pos[3 * i] - pos[3 * j], pos[3 * i + 1] - pos[3 * j + 1], pos[3 * i + 2] - pos[3 * j + 2],
                           true, Bp, tid);
            __syncthreads();
            for (int it = tid; it < P.nlm * P.nlm; it += nth) {
                int s = it / P.nlm, d = it - s * P.nlm;
                cplx Aa, Bb;
                combo_sums(P, s * P.nlm + d, Bp, Aa, Bb);
                cplx cp = cadd(Aa, Bb), cn = csub(Aa, Bb);
                const int lam = degree_of(d);
                const cplx* t4 = T + ((size_t)i * P.L + lam - 1) * 4;
                const int r0 = a * M + 2 * d, c0 = c * M + 2 * s;
                A[c0 * nb + r0] = cneg(cmul(t4[0], cp));
                A[c0 * nb + r0 + 1] = cneg(cmul(t4[2], cp));
                A[(c0 + 1) * nb + r0] = cneg(cmul(t4[1], cn));
                A[(c0 + 1) * nb + r0 + 1] = cneg(cmul(t4[3], cn));
            }
            __syncthreads();
        }
    if (!cta_lu(A, nb, piv, &sing)) {
        if (tid == 0) atomicExch(status, 5);
        return;
    }
    cplx* out = dinv + (size_t)b * PB_MAXMODES * PB_MAXMODES;
    for (int c0 = 0; c0 < nb; c0 += PB_PANEL) {
        const int nc = min(PB_PANEL, nb - c0);
        for (int t = tid; t < nb * nc; t += nth) {
            int jj = t / nb, r = t - jj * nb;
            Bp[jj * nb + r] = mk(r == c0 + jj ? 1.0 : 0.0, 0.0);
        }
        __syncthreads();
        cta_lu_solve(A, nb, piv, Bp, nc);
        for (int t = tid; t < nb * nc; t += nth) {
            int jj = t / nb, r = t - jj * nb;
            out[(size_t)(c0 + jj) * nb + r] = Bp[jj * nb + r];
        }
        __syncthreads();
    }
}

// y_b = Dinv_b x_b for every block; CTA per block, thread per row (fixed summation order)
__global__ void __launch_bounds__(128) blk_apply_kernel(int M, const int* __restrict__ bptr,
                                                        const int* __restrict__ bmem, const cplx* __restrict__ dinv,
                                                        const cplx* __restrict__ x, cplx* __restrict__ y) {
    __shared__ cplx xs[PB_MAXMODES];
    const int b = blockIdx.x;
    const int m0 = bptr[b], cnt = bptr[b + 1] - m0, nb = cnt * M;
    for (int r = threadIdx.x; r < nb; r += blockDim.x) xs[r] = x[(size_t)bmem[m0 + r / M] * M + r % M];
    __syncthreads();
    const cplx* D = dinv + (size_t)b * PB_MAXMODES * PB_MAXMODES;
    for (int r = threadIdx.x; r < nb; r += blockDim.x) {
        cplx acc = mk(0.0, 0.0);
        for (int c = 0; c < nb; ++c) cfma(acc, D[(size_t)c * nb + r], xs[c]);
        y[(size_t)bmem[m0 + r / M] * M + r % M] = acc;
    }
}

// Block Jacobi: spheres grouped into blocks of at most PB_MAXMODES modes, each block's own
// system (I - T C)_bb inverted exactly.
class BlockJacobiPre : public Preconditioner {
   public:
    int M = 0, nblocks = 0;
    int *d_bptr = nullptr, *d_bmem = nullptr;
    cplx* d_dinv = nullptr;
    DeviceAllocator *o_bptr = nullptr, *o_bmem = nullptr, *o_dinv = nullptr;
    long long* launches = nullptr;
    ~BlockJacobiPre() override {
        call_free(d_bptr, o_bptr);
        call_free(d_bmem, o_bmem);
        call_free(d_dinv, o_dinv);
    }
    void apply(const cplx* in, cplx* out, cudaStream_t st) override {
        blk_apply_kernel<<<nblocks, 128, 0, st>>>(M, d_bptr, d_bmem, d_dinv, in, out);
        if (launches) ++*launches;
    }
};

// One-sphere blocks (more than PB_MAXMODES modes per sphere): (I - T C)_ii = I, the identity.
class IdentityPre : public Preconditioner {
   public:
    size_t n = 0;
    void apply(const cplx* in, cplx* out, cudaStream_t st) override {
        cudaMemcpyAsync(out, in, n * sizeof(cplx), cudaMemcpyDeviceToDevice, st);
    }
};

}  // namespace

tcu_status make_block_jacobi(cudaStream_t st, const DevPlan& P, int N, double k0, const double* d_pos,
                             const double* h_pos, const double* h_radii, const double2* d_T,
                             std::unique_ptr<Preconditioner>* out, long long* launches) {
    if (2 * P.nlm > PB_MAXMODES) {
        auto id = std::make_unique<IdentityPre>();
        id->n = (size_t)N * 2 * P.nlm;
        *out = std::move(id);
        return TCU_OK;
    }
    auto pre = std::make_unique<BlockJacobiPre>();
    BlockJacobiPre& p = *pre;
    p.M = 2 * P.nlm;
    p.launches = launches;
    double rmax = 0.0;
    for (int i = 0; i < N; ++i) rmax = std::max(rmax, h_radii[i]);
    const int per_block = std::max(1, PB_MAXMODES / p.M);
    // blocks gather nearest neighbours within 3 sphere diameters
    Graph g = build_graph(N, h_pos, 6.0 * rmax, per_block);
    p.nblocks = (int)g.bptr.size() - 1;
    auto ck = [](cudaError_t e) { return e == cudaSuccess; };
    if (!ck(upload(&p.d_bptr, g.bptr, st, &p.o_bptr)) || !ck(upload(&p.d_bmem, g.bmem, st, &p.o_bmem)) ||
        !ck(call_malloc((void**)&p.d_dinv, (size_t)p.nblocks * PB_MAXMODES * PB_MAXMODES * sizeof(cplx), &p.o_dinv)))
        return TCU_OUT_OF_MEMORY;
    int* d_status = nullptr;
    DeviceAllocator* o_status = nullptr;
    if (!ck(call_malloc((void**)&d_status, sizeof(int), &o_status))) return TCU_OUT_OF_MEMORY;
    cudaMemsetAsync(d_status, 0, sizeof(int), st);
    size_t smem = (size_t)PB_MAXMODES * PB_MAXMODES * 16 + (size_t)PB_MAXMODES * PB_PANEL * 16;
    static PerDeviceOnce attr;
    once_per_device(attr, [&] {
        cudaFuncSetAttribute(blk_inverse_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    });
    blk_inverse_kernel<<<p.nblocks, 512, smem, st>>>(P, k0, d_pos, d_T, p.d_bptr, p.d_bmem, p.d_dinv, d_status);
    if (launches) ++*launches;
    int hst = 0;
    cudaMemcpyAsync(&hst, d_status, sizeof(int), cudaMemcpyDeviceToHost, st);
    cudaError_t e = cudaStreamSynchronize(st);
    call_free(d_status, o_status);
    if (e != cudaSuccess || cudaGetLastError() != cudaSuccess) return TCU_DEVICE_ERROR;
    if (hst == 5) return TCU_SINGULAR;
    *out = std::move(pre);
    return TCU_OK;
}

}  // namespace tcu
