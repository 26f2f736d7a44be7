// Right preconditioners of the matrix-free GMRES on A = I - T C (new here: the reference's
// iterative solver, cluster/iterative.rs:264-284 with linalg/gmres.rs:119, runs unpreconditioned).
//
// Both start from a split of the couplings by distance. Near-field pairs are those closer
// than `reach` sphere diameters (default: the reach of the compiled-in fit); their blocks K_ij = T_i C_ij are built once, stored as
// the helicity entries (A + B, A - B) of C_ij per (source lm, destination lm), and applied
// as a block-sparse product. Spheres are grouped into blocks of up to 96 modes
// (3 spheres at lmax 3, 2 at lmax 4): each sphere in Morton order that is still free opens
// a block and takes its nearest free neighbours.
//
//  * Block Jacobi: D = blockdiag((I - T C)_bb)^-1, the exact inverse of every block's own
//    system (one CTA per block: assembly, pivoted LU and inverse in shared memory).
//  * Learned: M = sum_k alpha_k (D N)^k D, k = 0..K, with N the near-field couplings between
//    different blocks. This is a K-layer linear message-passing network over the neighbour
//    graph whose messages are the physical translation blocks and whose layer weights
//    alpha_k are fitted on training clusters by least squares on ||(I - A M) v||^2 (the model
//    is linear in alpha, so the fit is exact; tcu_learned_precond_gram returns the Gram
//    matrix and right-hand side the fit needs). With alpha_k = 1 it is K block-Jacobi
//    relaxation sweeps on the near-field system (I - T C_near) y = v.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <numeric>
#include <vector>

#include "kernels.h"
#include "pairtable.cuh"
#include "precond.h"
#include "smem_lu.cuh"

namespace tcu {

// Fitted layer weights and near-field reach of the learned preconditioner (generated by
// treams_b200/train_precond.py; lmax without a fit falls back to alpha_k = 1).
#include "learned_coefficients.inc"

namespace {

constexpr int PB_MAXMODES = 96;  // modes per block (shared-memory LU)
constexpr int PB_PANEL = 48;

// ---- kernels ------------------------------------------------------------------------------
// Near-field blocks: CTA per Q consecutive neighbour entries; warp w builds the harmonic table
// of entry e0 + w, then thread (q, d) writes the helicity entries of every source s.
__global__ void __launch_bounds__(256) nf_block_kernel(DevPlan P, double k, const double* __restrict__ pos,
                                                       const int* __restrict__ row_of, const int* __restrict__ nbr,
                                                       int nnz, int Q, cplx* __restrict__ blocks) {
    extern __shared__ cplx nf_Z[];
    const int e0 = blockIdx.x * Q;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (int w = warp; w < Q; w += blockDim.x >> 5) {
        int e = e0 + w;
        if (e < nnz) {
            int i = row_of[e], j = nbr[e];
            pair_table(P, k, pos[3 * i] - pos[3 * j], pos[3 * i + 1] - pos[3 * j + 1], pos[3 * i + 2] - pos[3 * j + 2],
                       true, nf_Z + w * P.tsize, lane);
        }
    }
    __syncthreads();
    const int q = threadIdx.x / P.nlm, d = threadIdx.x - q * P.nlm;
    const int e = e0 + q;
    if (q >= Q || e >= nnz) return;
    const size_t nlm2 = (size_t)P.nlm * P.nlm;
    for (int s = 0; s < P.nlm; ++s) {
        cplx A, B;
        combo_sums(P, s * P.nlm + d, nf_Z + q * P.tsize, A, B);
        cplx* o = blocks + ((size_t)e * nlm2 + (size_t)s * P.nlm + d) * 2;
        o[0] = cadd(A, B);
        o[1] = csub(A, B);
    }
}

// y_i = zadd_i + T_i sum_{j in nb(i), skip[e] == 0} C_ij x_j; CTA per destination sphere,
// Q neighbour slots, fixed-order reduction over the slots.
__global__ void __launch_bounds__(256) nf_apply_kernel(int L, int nlm, const int* __restrict__ ptr,
                                                       const int* __restrict__ nbr, const uint8_t* __restrict__ skip,
                                                       const cplx* __restrict__ blocks, const cplx* __restrict__ T,
                                                       const cplx* __restrict__ x, const cplx* __restrict__ zadd,
                                                       cplx* __restrict__ y, int Q) {
    extern __shared__ cplx nf_red[];  // Q * nlm * 2
    const int i = blockIdx.x, M = 2 * nlm;
    const int q = threadIdx.x / nlm, d = threadIdx.x - q * nlm;
    const size_t nlm2 = (size_t)nlm * nlm;
    cplx ap = mk(0.0, 0.0), an = mk(0.0, 0.0);
    if (q < Q)
        for (int e = ptr[i] + q; e < ptr[i + 1]; e += Q) {
            if (skip[e]) continue;
            const cplx* bl = blocks + (size_t)e * nlm2 * 2;
            const cplx* xs = x + (size_t)nbr[e] * M;
            for (int s = 0; s < nlm; ++s) {
                cplx cp = bl[((size_t)s * nlm + d) * 2], cn = bl[((size_t)s * nlm + d) * 2 + 1];
                cfma(ap, cp, xs[2 * s]);
                cfma(an, cn, xs[2 * s + 1]);
            }
        }
    if (q < Q) {
        nf_red[(q * nlm + d) * 2] = ap;
        nf_red[(q * nlm + d) * 2 + 1] = an;
    }
    __syncthreads();
    for (int dd = threadIdx.x; dd < nlm; dd += blockDim.x) {
        cplx sp = mk(0.0, 0.0), sn = mk(0.0, 0.0);
        for (int qq = 0; qq < Q; ++qq) {
            sp = cadd(sp, nf_red[(qq * nlm + dd) * 2]);
            sn = cadd(sn, nf_red[(qq * nlm + dd) * 2 + 1]);
        }
        const int lam = degree_of(dd);
        const cplx* t4 = T + ((size_t)i * L + lam - 1) * 4;
        cplx y0 = cadd(cmul(t4[0], sp), cmul(t4[1], sn));
        cplx y1 = cadd(cmul(t4[2], sp), cmul(t4[3], sn));
        size_t row = (size_t)i * M + 2 * dd;
        if (zadd) {
            y0 = cadd(y0, zadd[row]);
            y1 = cadd(y1, zadd[row + 1]);
        }
        y[row] = y0;
        y[row + 1] = y1;
    }
}

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

// ---- host set-up ----------------------------------------------------------------------------
uint64_t spread3(uint64_t v) {  // 21 bits -> every third bit
    v &= 0x1fffff;
    v = (v | v << 32) & 0x1f00000000ffffULL;
    v = (v | v << 16) & 0x1f0000ff0000ffULL;
    v = (v | v << 8) & 0x100f00f00f00f00fULL;
    v = (v | v << 4) & 0x10c30c30c30c30c3ULL;
    v = (v | v << 2) & 0x1249249249249249ULL;
    return v;
}

struct Graph {
    std::vector<int> ptr, nbr, row_of, bptr, bmem, block_of;
    std::vector<uint8_t> same;
};

// Neighbours within `reach` (sorted by index) and blocks of at most `per_block` spheres.
Graph build_graph(int N, const double* pos, double reach, int per_block) {
    Graph g;
    double lo[3] = {1e300, 1e300, 1e300};
    for (int i = 0; i < N; ++i)
        for (int a = 0; a < 3; ++a) lo[a] = std::min(lo[a], pos[3 * i + a]);
    auto cell = [&](int i, int a) { return (long)std::floor((pos[3 * i + a] - lo[a]) / reach); };
    std::vector<std::pair<uint64_t, int>> order(N);
    for (int i = 0; i < N; ++i)
        order[i] = {spread3(cell(i, 0)) | spread3(cell(i, 1)) << 1 | spread3(cell(i, 2)) << 2, i};
    std::sort(order.begin(), order.end());
    // cell lists in Morton order: spheres sharing a cell are contiguous
    std::vector<std::vector<int>> nb(N);
    {
        long dim = 1;
        for (int i = 0; i < N; ++i)
            for (int a = 0; a < 3; ++a) dim = std::max(dim, cell(i, a) + 2);
        std::vector<std::pair<long, int>> byc(N);
        for (int i = 0; i < N; ++i) byc[i] = {(cell(i, 0) * dim + cell(i, 1)) * dim + cell(i, 2), i};
        std::sort(byc.begin(), byc.end());
        for (int i = 0; i < N; ++i) {
            long cx = cell(i, 0), cy = cell(i, 1), cz = cell(i, 2);
            for (long dx = -1; dx <= 1; ++dx)
                for (long dy = -1; dy <= 1; ++dy)
                    for (long dz = -1; dz <= 1; ++dz) {
                        long x = cx + dx, y = cy + dy, z = cz + dz;
                        if (x < 0 || y < 0 || z < 0) continue;
                        long key = (x * dim + y) * dim + z;
                        auto it = std::lower_bound(byc.begin(), byc.end(), std::make_pair(key, -1));
                        for (; it != byc.end() && it->first == key; ++it) {
                            int j = it->second;
                            if (j == i) continue;
                            double d = std::hypot(std::hypot(pos[3 * i] - pos[3 * j], pos[3 * i + 1] - pos[3 * j + 1]),
                                                  pos[3 * i + 2] - pos[3 * j + 2]);
                            if (d <= reach) nb[i].push_back(j);
                        }
                    }
            std::sort(nb[i].begin(), nb[i].end());
        }
    }
    // blocks: each free sphere in Morton order takes its nearest free neighbours
    g.block_of.assign(N, -1);
    g.bptr.push_back(0);
    for (auto& o : order) {
        int i = o.second;
        if (g.block_of[i] >= 0) continue;
        int b = (int)g.bptr.size() - 1;
        g.block_of[i] = b;
        g.bmem.push_back(i);
        std::vector<std::pair<double, int>> cand;
        for (int j : nb[i])
            if (g.block_of[j] < 0)
                cand.push_back({std::hypot(std::hypot(pos[3 * i] - pos[3 * j], pos[3 * i + 1] - pos[3 * j + 1]),
                                           pos[3 * i + 2] - pos[3 * j + 2]),
                                j});
        std::sort(cand.begin(), cand.end());
        for (size_t c = 0; c < cand.size() && (int)(g.bmem.size() - g.bptr.back()) < per_block; ++c) {
            g.block_of[cand[c].second] = b;
            g.bmem.push_back(cand[c].second);
        }
        g.bptr.push_back((int)g.bmem.size());
    }
    g.ptr.assign(N + 1, 0);
    for (int i = 0; i < N; ++i) {
        g.ptr[i + 1] = g.ptr[i] + (int)nb[i].size();
        for (int j : nb[i]) {
            g.nbr.push_back(j);
            g.row_of.push_back(i);
            g.same.push_back(g.block_of[i] == g.block_of[j] ? 1 : 0);
        }
    }
    return g;
}

template <typename T>
cudaError_t upload(T** d, const std::vector<T>& h, cudaStream_t st) {
    cudaError_t e = cudaMalloc((void**)d, std::max<size_t>(h.size(), 1) * sizeof(T));
    if (e != cudaSuccess) return e;
    if (!h.empty()) e = cudaMemcpyAsync(*d, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice, st);
    return e;
}

class NearFieldPre : public Preconditioner {
   public:
    int L = 0, nlm = 0, M = 0, N = 0, nblocks = 0, layers = 0;
    size_t n = 0, nnz = 0;
    const cplx* T = nullptr;  // caller-owned Mie blocks
    int *d_ptr = nullptr, *d_nbr = nullptr, *d_row = nullptr, *d_bptr = nullptr, *d_bmem = nullptr;
    uint8_t* d_same = nullptr;
    cplx *d_blocks = nullptr, *d_dinv = nullptr, *d_basis = nullptr, *d_tmp = nullptr, *d_alpha = nullptr;
    long long* launches = nullptr;
    ~NearFieldPre() override {
        for (void* p : {(void*)d_ptr, (void*)d_nbr, (void*)d_row, (void*)d_bptr, (void*)d_bmem, (void*)d_same,
                        (void*)d_blocks, (void*)d_dinv, (void*)d_basis, (void*)d_tmp, (void*)d_alpha})
            if (p) cudaFree(p);
    }
    void block_apply(const cplx* in, cplx* out, cudaStream_t st) {
        blk_apply_kernel<<<nblocks, 128, 0, st>>>(M, d_bptr, d_bmem, d_dinv, in, out);
        if (launches) ++*launches;
    }
    // out = T (C_near, other blocks) in
    void near_apply(const cplx* in, cplx* out, cudaStream_t st) {
        int Q = std::min(16, 256 / nlm);
        nf_apply_kernel<<<N, 256, (size_t)Q * nlm * 2 * sizeof(cplx), st>>>(L, nlm, d_ptr, d_nbr, d_same, d_blocks, T, in,
                                                                           nullptr, out, Q);
        if (launches) ++*launches;
    }
    // basis s_0 = D v, s_k = D N s_(k-1), k <= layers, into d_basis (layers + 1 vectors)
    void basis(const cplx* in, cudaStream_t st) {
        block_apply(in, d_basis, st);
        for (int kk = 1; kk <= layers; ++kk) {
            near_apply(d_basis + (size_t)(kk - 1) * n, d_tmp, st);
            block_apply(d_tmp, d_basis + (size_t)kk * n, st);
        }
    }
    void apply(const cplx* in, cplx* out, cudaStream_t st) override {
        if (layers == 0) {
            block_apply(in, out, st);
            return;
        }
        basis(in, st);
        cudaMemsetAsync(out, 0, n * sizeof(cplx), st);
        vec_lincomb(out, d_basis, n, layers + 1, d_alpha, n, st);
        if (launches) ++*launches;
    }
};

tcu_status build_nearfield(cudaStream_t st, const DevPlan& P, int L, int N, double k0, const double* d_pos,
                           const double* h_pos, const double* h_radii, const cplx* d_T, double reach, int layers,
                           const std::vector<std::complex<double>>& alpha, std::unique_ptr<NearFieldPre>* out,
                           long long* launches) {
    auto pre = std::make_unique<NearFieldPre>();
    NearFieldPre& p = *pre;
    p.L = L;
    p.nlm = P.nlm;
    p.M = 2 * P.nlm;
    p.N = N;
    p.n = (size_t)N * p.M;
    p.T = d_T;
    p.layers = layers;
    p.launches = launches;
    double rmax = 0.0;
    for (int i = 0; i < N; ++i) rmax = std::max(rmax, h_radii[i]);
    int per_block = std::max(1, PB_MAXMODES / p.M);
    Graph g = build_graph(N, h_pos, 2.0 * (reach > 0.0 ? reach : LEARNED_REACH) * rmax, per_block);
    p.nnz = g.nbr.size();
    p.nblocks = (int)g.bptr.size() - 1;
    auto ck = [](cudaError_t e) { return e == cudaSuccess; };
    if (!ck(upload(&p.d_ptr, g.ptr, st)) || !ck(upload(&p.d_nbr, g.nbr, st)) || !ck(upload(&p.d_row, g.row_of, st)) ||
        !ck(upload(&p.d_same, g.same, st)) || !ck(upload(&p.d_bptr, g.bptr, st)) ||
        !ck(upload(&p.d_bmem, g.bmem, st)))
        return TCU_OUT_OF_MEMORY;
    size_t nlm2 = (size_t)p.nlm * p.nlm;
    const size_t nblk_entries = layers > 0 ? std::max<size_t>(p.nnz, 1) : 1;  // block Jacobi needs no near field
    if (!ck(cudaMalloc((void**)&p.d_blocks, nblk_entries * nlm2 * 2 * sizeof(cplx))) ||
        !ck(cudaMalloc((void**)&p.d_dinv, (size_t)p.nblocks * PB_MAXMODES * PB_MAXMODES * sizeof(cplx))) ||
        !ck(cudaMalloc((void**)&p.d_basis, (size_t)(layers + 1) * p.n * sizeof(cplx))) ||
        !ck(cudaMalloc((void**)&p.d_tmp, p.n * sizeof(cplx))) ||
        !ck(cudaMalloc((void**)&p.d_alpha, (size_t)(layers + 1) * sizeof(cplx))))
        return TCU_OUT_OF_MEMORY;
    std::vector<cplx> a(layers + 1);
    for (int kk = 0; kk <= layers; ++kk)
        a[kk] = mk(kk < (int)alpha.size() ? alpha[kk].real() : 1.0, kk < (int)alpha.size() ? alpha[kk].imag() : 0.0);
    cudaMemcpyAsync(p.d_alpha, a.data(), a.size() * sizeof(cplx), cudaMemcpyHostToDevice, st);
    int* d_status = nullptr;
    if (!ck(cudaMalloc((void**)&d_status, sizeof(int)))) return TCU_OUT_OF_MEMORY;
    cudaMemsetAsync(d_status, 0, sizeof(int), st);
    if (p.nnz > 0 && layers > 0) {
        int Q = std::min(16, 256 / p.nlm);
        unsigned grid = (unsigned)((p.nnz + Q - 1) / Q);
        nf_block_kernel<<<grid, 256, (size_t)Q * P.tsize * sizeof(cplx), st>>>(P, k0, d_pos, p.d_row, p.d_nbr,
                                                                               (int)p.nnz, Q, p.d_blocks);
        if (launches) ++*launches;
    }
    size_t smem = (size_t)PB_MAXMODES * PB_MAXMODES * 16 + (size_t)PB_MAXMODES * PB_PANEL * 16;
    cudaFuncSetAttribute(blk_inverse_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    blk_inverse_kernel<<<p.nblocks, 512, smem, st>>>(P, k0, d_pos, d_T, p.d_bptr, p.d_bmem, p.d_dinv, d_status);
    if (launches) ++*launches;
    int hst = 0;
    cudaMemcpyAsync(&hst, d_status, sizeof(int), cudaMemcpyDeviceToHost, st);
    cudaError_t e = cudaStreamSynchronize(st);
    cudaFree(d_status);
    if (e != cudaSuccess || cudaGetLastError() != cudaSuccess) return TCU_DEVICE_ERROR;
    if (hst == 5) return TCU_SINGULAR;
    *out = std::move(pre);
    return TCU_OK;
}

}  // namespace

tcu_status make_preconditioner(cudaStream_t st, int kind, const DevPlan& P, int L, int N, double k0,
                               const double* d_pos, const double* h_pos, const double* h_radii, const double2* d_T,
                               double reach, int layers_in, const std::vector<std::complex<double>>& alpha_in,
                               std::unique_ptr<Preconditioner>* out, long long* launches) {
    std::unique_ptr<NearFieldPre> pre;
    std::vector<std::complex<double>> alpha;
    int layers = 0;
    if (kind == TCU_PRECOND_LEARNED) {
        if (layers_in < 0) {
            layers = LEARNED_LAYERS;
            for (int kk = 0; kk <= layers; ++kk) alpha.push_back(learned_alpha(L, kk));
        } else {
            layers = layers_in;
            alpha = alpha_in;
        }
    }
    tcu_status s =
        build_nearfield(st, P, L, N, k0, d_pos, h_pos, h_radii, d_T, reach, layers, alpha, &pre, launches);
    if (s) return s;
    *out = std::move(pre);
    return TCU_OK;
}

tcu_status learned_gram(cudaStream_t st, const DevPlan& P, int L, int N, double k0, const double* d_pos,
                        const double* h_pos, const double* h_radii, const double2* d_T, double reach, int layers,
                        int nvec,
                        const double2* d_V, double2* d_gram_scratch, double2* d_partial, std::complex<double>* gram,
                        std::complex<double>* rhs, long long* launches) {
    std::unique_ptr<NearFieldPre> pre;
    std::vector<std::complex<double>> alpha(layers + 1, 1.0);
    tcu_status s =
        build_nearfield(st, P, L, N, k0, d_pos, h_pos, h_radii, d_T, reach, layers, alpha, &pre, launches);
    if (s) return s;
    const size_t n = pre->n;
    const int K1 = layers + 1;
    cplx* U = nullptr;
    if (cudaMalloc((void**)&U, (size_t)K1 * n * sizeof(cplx)) != cudaSuccess) return TCU_OUT_OF_MEMORY;
    std::vector<cplx> col(K1);
    for (int i = 0; i < K1 * K1; ++i) gram[i] = 0.0;
    for (int i = 0; i < K1; ++i) rhs[i] = 0.0;
    for (int v = 0; v < nvec; ++v) {
        const cplx* vin = d_V + (size_t)v * n;
        pre->basis(vin, st);
        for (int kk = 0; kk < K1; ++kk) {  // u_k = A s_k
            launch_apply(P, N, k0, d_pos, d_T, pre->d_basis + (size_t)kk * n, n, 1, nullptr, 1.0, -1.0, true,
                         U + (size_t)kk * n, st);
            if (launches) ++*launches;
        }
        for (int l = 0; l <= K1; ++l) {  // columns of U^H U, then U^H v
            const cplx* w = l < K1 ? U + (size_t)l * n : vin;
            vec_dots(U, n, K1, w, n, d_gram_scratch, d_partial, st);
            cudaMemcpyAsync(col.data(), d_gram_scratch, K1 * sizeof(cplx), cudaMemcpyDeviceToHost, st);
            if (cudaStreamSynchronize(st) != cudaSuccess) {
                cudaFree(U);
                return TCU_DEVICE_ERROR;
            }
            for (int kk = 0; kk < K1; ++kk) {
                std::complex<double> c(col[kk].x, col[kk].y);
                if (l < K1)
                    gram[kk * K1 + l] += c;  // row k, column l: conj(u_k) . u_l
                else
                    rhs[kk] += c;
            }
            if (launches) *launches += 2;
        }
    }
    cudaFree(U);
    return cudaGetLastError() == cudaSuccess ? TCU_OK : TCU_DEVICE_ERROR;
}

}  // namespace tcu
