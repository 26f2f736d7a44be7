// Near-field couplings shared by the GMRES preconditioners (precond.cu, gnn.cu): the
// neighbour graph of a cluster (pairs closer than a reach, cell lists in Morton order, blocks
// of nearest neighbours), the blocks C_ij of the near-field pairs stored as helicity entries
// (A + B, A - B) per (source lm, destination lm), and their block-sparse product with T.
#pragma once
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <vector>

#include "kernels.h"
#include "pairtable.cuh"

namespace tcu {
namespace nearfield {
namespace {  // internal linkage: every including file keeps its own copy

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

// squared distance of sphere centres (plain arithmetic: centres are finite and well inside the
// double range, validated on entry)
inline double dist2(const double* pos, int i, int j) {
    const double dx = pos[3 * i] - pos[3 * j], dy = pos[3 * i + 1] - pos[3 * j + 1], dz = pos[3 * i + 2] - pos[3 * j + 2];
    return dx * dx + dy * dy + dz * dz;
}

// Neighbours within `reach` (sorted by index) and blocks of at most `per_block` spheres.
// Cells of side `reach`; spheres sorted by cell, each cell's range found in a dense table
// (or by binary search when the grid is much larger than the cluster); neighbour lists are
// written straight into CSR.
Graph build_graph(int N, const double* pos, double reach, int per_block) {
    Graph g;
    const double reach2 = reach * reach;
    double lo[3] = {1e300, 1e300, 1e300};
    for (int i = 0; i < N; ++i)
        for (int a = 0; a < 3; ++a) lo[a] = std::min(lo[a], pos[3 * i + a]);
    std::vector<long> cc(3 * (size_t)N);
    long dim = 1;
    for (int i = 0; i < N; ++i)
        for (int a = 0; a < 3; ++a) {
            cc[3 * i + a] = (long)std::floor((pos[3 * i + a] - lo[a]) / reach);
            dim = std::max(dim, cc[3 * i + a] + 2);
        }
    std::vector<std::pair<uint64_t, int>> order(N);
    for (int i = 0; i < N; ++i)
        order[i] = {spread3(cc[3 * i]) | spread3(cc[3 * i + 1]) << 1 | spread3(cc[3 * i + 2]) << 2, i};
    std::sort(order.begin(), order.end());
    auto key_of = [&](long x, long y, long z) { return (x * dim + y) * dim + z; };
    std::vector<std::pair<long, int>> byc(N);
    for (int i = 0; i < N; ++i) byc[i] = {key_of(cc[3 * i], cc[3 * i + 1], cc[3 * i + 2]), i};
    std::sort(byc.begin(), byc.end());
    const bool dense = dim <= 4096 && dim * dim * dim <= 8L * N + 4096;
    std::vector<int> cstart;
    if (dense) {
        cstart.assign((size_t)(dim * dim * dim) + 1, 0);
        for (const auto& e : byc) ++cstart[(size_t)e.first + 1];
        for (size_t k = 1; k < cstart.size(); ++k) cstart[k] += cstart[k - 1];
    }
    g.ptr.assign(N + 1, 0);
    std::vector<int> tmp;
    for (int i = 0; i < N; ++i) {
        tmp.clear();
        const long cx = cc[3 * i], cy = cc[3 * i + 1], cz = cc[3 * i + 2];
        for (long dx = -1; dx <= 1; ++dx)
            for (long dy = -1; dy <= 1; ++dy)
                for (long dz = -1; dz <= 1; ++dz) {
                    const long x = cx + dx, y = cy + dy, z = cz + dz;
                    if (x < 0 || y < 0 || z < 0 || x >= dim || y >= dim || z >= dim) continue;
                    const long key = key_of(x, y, z);
                    size_t b0, b1;
                    if (dense) {
                        b0 = (size_t)cstart[(size_t)key];
                        b1 = (size_t)cstart[(size_t)key + 1];
                    } else {
                        b0 = std::lower_bound(byc.begin(), byc.end(), std::make_pair(key, -1)) - byc.begin();
                        b1 = b0;
                        while (b1 < byc.size() && byc[b1].first == key) ++b1;
                    }
                    for (size_t q = b0; q < b1; ++q) {
                        const int j = byc[q].second;
                        if (j != i && dist2(pos, i, j) <= reach2) tmp.push_back(j);
                    }
                }
        std::sort(tmp.begin(), tmp.end());
        g.nbr.insert(g.nbr.end(), tmp.begin(), tmp.end());
        g.row_of.insert(g.row_of.end(), tmp.size(), i);
        g.ptr[i + 1] = (int)g.nbr.size();
    }
    // blocks: each free sphere in Morton order takes its nearest free neighbours
    g.block_of.assign(N, -1);
    g.bptr.push_back(0);
    std::vector<std::pair<double, int>> cand;
    for (auto& o : order) {
        int i = o.second;
        if (g.block_of[i] >= 0) continue;
        int b = (int)g.bptr.size() - 1;
        g.block_of[i] = b;
        g.bmem.push_back(i);
        if (per_block > 1) {
            cand.clear();
            for (int e = g.ptr[i]; e < g.ptr[i + 1]; ++e) {
                const int j = g.nbr[e];
                if (g.block_of[j] < 0) cand.push_back({dist2(pos, i, j), j});
            }
            std::sort(cand.begin(), cand.end());
            for (size_t c = 0; c < cand.size() && (int)(g.bmem.size() - g.bptr.back()) < per_block; ++c) {
                g.block_of[cand[c].second] = b;
                g.bmem.push_back(cand[c].second);
            }
        }
        g.bptr.push_back((int)g.bmem.size());
    }
    g.same.resize(g.nbr.size());
    for (size_t e = 0; e < g.nbr.size(); ++e) g.same[e] = g.block_of[g.row_of[e]] == g.block_of[g.nbr[e]] ? 1 : 0;
    return g;
}

template <typename T>
cudaError_t upload(T** d, const std::vector<T>& h, cudaStream_t st, DeviceAllocator** owner) {
    cudaError_t e = call_malloc((void**)d, std::max<size_t>(h.size(), 1) * sizeof(T), owner);
    if (e != cudaSuccess) return e;
    if (!h.empty()) e = cudaMemcpyAsync(*d, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice, st);
    return e;
}


}  // namespace
}  // namespace nearfield
}  // namespace tcu
