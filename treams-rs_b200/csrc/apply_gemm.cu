// Matrix-free operator x - T C x in product form, for lmax 2..5, and its dipole blocks (any
// lmax): the columns of the dipole sources (the coarse correction of the two-level
// preconditioner) and the dipole-to-dipole block (its coarse operator).
//
// The coupling of destination sphere i is, per destination mode d and helicity,
//   (C x)_i[d, +] = sum_{j != i} sum_s (A_ij(s,d) + B_ij(s,d)) x_j[2s]
//   (C x)_i[d, -] = sum_{j != i} sum_s (A_ij(s,d) - B_ij(s,d)) x_j[2s+1]
// with A and B the plan's term sums over the pair's harmonic table Z_ij (sw/plan.rs:224-251,
// sw/coupling.rs:127-140). Exchanging the sums over j and over the plan's terms gives
//   G_i[idx, e] = sum_{j != i} Z_ij[idx] x_j[e]            (tsize x 2 nlm per destination)
//   (C x)_i[d, +] = sum_s sum_{t in A(s,d) + B(s,d)} w_t G_i[idx_t, 2s]   (and - for B at 2s+1)
// The first line is a complex product of the generated table matrix Z_i (tsize x N) with the
// coefficients X (N x 2 nlm): a register-tiled FP64 product whose A operand is built in shared
// memory chunk by chunk and never stored. The plan's term lists then run once per destination
// instead of once per pair. Work per ordered pair: tsize * 2 nlm complex multiply-adds
// (1,470 at lmax 3, 3,888 at lmax 4) plus one harmonic table.
//
// CTA = DI destination spheres x one right-hand side, RG x CG threads; thread (rg, cg) owns
// G rows rg + RG u (u < TR) and columns cg + CG t (t < TC). Per chunk of KJ sources:
//   A) thread per pair: direction and radial sequence z_p(k r), p <= 2 lmax, to shared memory;
//   B) thread per (pair, order m >= 0): the order column of the solid harmonics times z_p,
//      written into the chunk's table matrix (rows dest * tsize + idx, one column per source);
//   C) the chunk's product update from shared memory.
// Finally G goes to shared memory and thread per (destination, d) applies the term lists,
// the Mie block and the alpha / beta / zadd epilogue of the operator.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdlib>
#include <cstring>

#include "common.cuh"
#include "kernels.h"
#include "pairtable.cuh"
#include "plan.h"

namespace tcu {

namespace {

struct GemmShape {
    int DI, TR, TC, RG, CG, KJ;
};

// The product restricted to the first nsrc source lm and the first ndst destination lm (the
// table then needs degrees p <= order = l_max(src) + l_max(dst)); input vectors hold ldin and
// output vectors ldout complex entries per sphere. The full operator: nsrc = ndst = nlm.
struct SubOp {
    int nsrc, ndst, order, ldin, ldout;
};

// Tile shapes per lmax: G rows DI * tsize <= TR * RG, columns 2 nlm <= TC * CG
GemmShape gemm_shape(int L) {
    switch (L) {
        case 2: return {4, 4, 2, 25, 8, 32};   // 100 x 16, 200 threads
        case 3: return {2, 4, 3, 25, 10, 32};  // 98 x 30, 250 threads
        case 4: return {1, 4, 4, 21, 12, 32};  // 81 x 48, 252 threads
        default: return {1, 4, 5, 31, 14, 16}; // lmax 5: 121 x 70, 434 threads
    }
}

// The dipole-source (and dipole-to-dipole) products: G is (DI (order+1)^2) x 6, about 200 rows
GemmShape sub_shape(int tsz) {
    const int DI = std::max(1, 200 / tsz);
    return {DI, 4, 2, (DI * tsz + 3) / 4, 3, 16};
}

size_t gemm_smem(const SubOp& o, const GemmShape& s) {
    const size_t tsz = (size_t)(o.order + 1) * (o.order + 1);
    const size_t rows = (size_t)s.TR * s.RG + 1, cols = (size_t)s.TC * s.CG, npair = (size_t)s.DI * s.KJ;
    const size_t chunk = ((size_t)s.KJ * rows + (size_t)s.KJ * cols + npair * (o.order + 1)) * sizeof(cplx) +
                         npair * sizeof(double4);
    const size_t g = (size_t)s.DI * tsz * 2 * o.nsrc * sizeof(cplx);
    return chunk > g ? chunk : g;
}

// Phases A and B of one chunk: the harmonic tables of the pairs (i0 + il, j0 + jj), il < DI,
// jj < KJ, into Zs (row il * ts + idx, column jj, leading dimension ZLD); Rs and Ds hold the
// radial sequences and directions. One barrier inside (between A and B), none at the end.
__device__ __forceinline__ void build_chunk(const DevPlan& P, int order, int N, double k,
                                            const double* __restrict__ pos, bool singular, int i0, int j0,
                                            int DI, int KJ, int ZLD, cplx* Zs, cplx* Rs, double4* Ds, int tid,
                                            int nthr) {
    const int ord1 = order + 1, ts = ord1 * ord1, npair = DI * KJ;
    // A) per pair: state 2 = a table, 1 = coincident centres of the regular kind (Z = e_0),
    //    0 = no coupling (the pair i = j, sources or destinations past N, coincident outgoing)
    for (int p = tid; p < npair; p += nthr) {
        const int il = p / KJ, jj = p - il * KJ, i = i0 + il, j = j0 + jj;
        double u[3] = {0.0, 0.0, 0.0}, state = 0.0;
        if (i < N && j < N && j != i) {
            double r;
            if (unit_direction(pos[3 * i] - pos[3 * j], pos[3 * i + 1] - pos[3 * j + 1],
                               pos[3 * i + 2] - pos[3 * j + 2], r, u)) {
                state = 2.0;
                cplx* rad = Rs + (size_t)p * ord1;
                if (singular) {
                    cplx h[MAXP];
                    hankel_sequence<MAXP>(order, k * r, h);
                    for (int q = 0; q <= order; ++q) rad[q] = h[q];
                } else {
                    double jv[MAXP];
                    bessel_j_sequence<MAXP>(order, k * r, jv);
                    for (int q = 0; q <= order; ++q) rad[q] = mk(jv[q], 0.0);
                }
            } else if (!singular) {
                state = 1.0;
            }
        }
        Ds[p] = make_double4(u[0], u[1], u[2], state);
    }
    __syncthreads();
    // B) per (pair, order m >= 0): column m of the table, entries deg = m..order at
    //    deg^2 + deg + m and deg^2 + deg - m
    for (int it = tid; it < npair * ord1; it += nthr) {
        const int p = it / ord1, m = it - p * ord1;
        const int il = p / KJ, jj = p - il * KJ;
        cplx* Zp = Zs + (size_t)jj * ZLD + (size_t)il * ts;
        const double4 D = Ds[p];
        if (D.w == 2.0) {
            const cplx* rad = Rs + (size_t)p * ord1;
            const cplx xy = mk(D.x, D.y);
            const double z = D.z, r2 = D.x * D.x + D.y * D.y + D.z * D.z;
            cplx diag = mk(1.0, 0.0);
            for (int q = 1; q <= m; ++q) diag = cscale(cmul(diag, xy), -double(2 * q - 1));
            cplx pc = diag, prev = mk(0.0, 0.0);
            for (int deg = m; deg <= order; ++deg) {
                if (deg > m) {
                    const double a = double(2 * deg - 1) / double(deg - m);
                    const double b = double(deg + m - 1) / double(deg - m);
                    const cplx next = mk(a * z * pc.x - b * r2 * prev.x, a * z * pc.y - b * r2 * prev.y);
                    prev = pc;
                    pc = next;
                }
                const cplx rd = rad[deg];
                Zp[deg * deg + deg + m] = cmul(rd, pc);
                if (m > 0) {
                    const int idx = deg * deg + deg - m;
                    Zp[idx] = cmul(rd, cscale(cconj(pc), P.reflection[idx]));
                }
            }
        } else {
            for (int deg = m; deg <= order; ++deg) {
                Zp[deg * deg + deg + m] = mk((D.w == 1.0 && deg == 0) ? 1.0 : 0.0, 0.0);
                if (m > 0) Zp[deg * deg + deg - m] = mk(0.0, 0.0);
            }
        }
    }
}

// Term lists of the plan, Mie block and the alpha / beta / zadd epilogue: thread per
// (destination, d) of the DI destinations from i0, with G of destination il at
// Gs + il * tsize * 2 nsrc (rows: table index, columns: source lm and helicity).
__device__ __forceinline__ void terms_epilogue(const DevPlan& P, const SubOp& O, const cplx* Gs, int DI, int i0,
                                               int N, const cplx* __restrict__ T, const cplx* __restrict__ xc,
                                               size_t coff, const cplx* __restrict__ zadd, double alpha,
                                               double beta, bool singular, cplx* __restrict__ y, int tid,
                                               int nthr) {
    const int nlm = P.nlm, M = 2 * O.nsrc, ts = (O.order + 1) * (O.order + 1);
    const int ndst = O.ndst;
    for (int it = tid; it < DI * ndst; it += nthr) {
        const int il = it / ndst, d = it - il * ndst, i = i0 + il;
        if (i >= N) continue;
        const cplx* G = Gs + (size_t)il * ts * M;
        cplx sp = mk(0.0, 0.0), sn = mk(0.0, 0.0);
        for (int s = 0; s < O.nsrc; ++s) {
            const int2 cb = __ldg(&P.combo[s * nlm + d]);
            int t = cb.x;
            const int na = cb.y & 0xffff, nb = cb.y >> 16;
            const cplx* g = G + 2 * s;
            for (int e = 0; e < na; ++e, ++t) {
                const cplx w = __ldg(&P.w[t]);
                const cplx* ge = g + (size_t)__ldg(&P.idx[t]) * M;
                cfma(sp, w, ge[0]);
                cfma(sn, w, ge[1]);
            }
            for (int e = 0; e < nb; ++e, ++t) {
                const cplx w = __ldg(&P.w[t]);
                const cplx* ge = g + (size_t)__ldg(&P.idx[t]) * M;
                cfma(sp, w, ge[0]);
                cfma(sn, cneg(w), ge[1]);
            }
        }
        // the input at (i, d) exists for source lm only (d < nsrc), the output for d < ndst
        const size_t row = (size_t)i * O.ldout + 2 * d, rin = (size_t)i * O.ldin + 2 * d;
        const cplx x0 = d < O.nsrc ? xc[rin] : mk(0.0, 0.0), x1 = d < O.nsrc ? xc[rin + 1] : mk(0.0, 0.0);
        cplx y0, y1;
        if (singular) {
            cplx tc0 = sp, tc1 = sn;  // T null: the coupling alone
            if (T) {
                const int lam = degree_of(d);
                const cplx* t4 = T + ((size_t)i * P.L + lam - 1) * 4;
                tc0 = cadd(cmul(t4[0], sp), cmul(t4[1], sn));
                tc1 = cadd(cmul(t4[2], sp), cmul(t4[3], sn));
            }
            y0 = cadd(cscale(x0, alpha), cscale(tc0, beta));
            y1 = cadd(cscale(x1, alpha), cscale(tc1, beta));
            if (zadd) {
                y0 = cadd(y0, zadd[coff + row]);
                y1 = cadd(y1, zadd[coff + row + 1]);
            }
        } else {
            y0 = cadd(x0, sp);
            y1 = cadd(x1, sn);
        }
        y[coff + row] = y0;
        y[coff + row + 1] = y1;
    }
}

template <int TR, int TC>
__global__ void __launch_bounds__(512, 1)
    apply_gemm_kernel(DevPlan P, SubOp O, int N, double k, const double* __restrict__ pos, const cplx* __restrict__ T,
                      const cplx* __restrict__ x, size_t ldx, const cplx* __restrict__ zadd, double alpha, double beta,
                      bool singular, cplx* __restrict__ y, int DI, int RG, int CG, int KJ) {
    extern __shared__ __align__(16) unsigned char ag_smem[];
    const int M = 2 * O.nsrc, order = O.order, ord1 = order + 1, ts = ord1 * ord1;
    // ZLD = ROWS + 1: the builder's writes of different sources (one column each) fall into
    // different banks; the product reads consecutive rows of one column
    const int ROWS = TR * RG, ZLD = ROWS + 1, COLS = TC * CG, npair = DI * KJ;
    cplx* Zs = reinterpret_cast<cplx*>(ag_smem);                     // KJ x ZLD (source-major)
    cplx* Xs = Zs + (size_t)KJ * ZLD;                                // KJ x COLS
    cplx* Rs = Xs + (size_t)KJ * COLS;                               // npair x (order + 1)
    double4* Ds = reinterpret_cast<double4*>(Rs + (size_t)npair * ord1);  // direction, state
    cplx* Gs = reinterpret_cast<cplx*>(ag_smem);                     // at the end: DI * ts x M
    const int tid = threadIdx.x, nthr = blockDim.x;
    const int rg = tid / CG, cg = tid - (tid / CG) * CG;
    const bool worker = rg < RG;
    const int i0 = blockIdx.x * DI;
    const size_t coff = (size_t)blockIdx.y * ldx;  // column offset, input and output alike
    const cplx* xc = x + coff;

    cplx acc[TR][TC];
#pragma unroll
    for (int u = 0; u < TR; ++u)
#pragma unroll
        for (int t = 0; t < TC; ++t) acc[u][t] = mk(0.0, 0.0);
    for (int t = tid; t < KJ * ZLD; t += nthr) Zs[t] = mk(0.0, 0.0);  // padding rows stay zero

    for (int j0 = 0; j0 < N; j0 += KJ) {
        __syncthreads();  // the previous chunk's product is done with Zs / Xs
        for (int t = tid; t < KJ * COLS; t += nthr) {
            const int jj = t / COLS, col = t - jj * COLS, j = j0 + jj;
            Xs[t] = (col < M && j < N) ? xc[(size_t)j * O.ldin + col] : mk(0.0, 0.0);
        }
        build_chunk(P, order, N, k, pos, singular, i0, j0, DI, KJ, ZLD, Zs, Rs, Ds, tid, nthr);
        __syncthreads();
        // C) G += Z_chunk X_chunk
        if (worker) {
            const cplx* zr = Zs + rg;
            const cplx* xr = Xs + cg;
            for (int kk = 0; kk < KJ; ++kk) {
                cplx a[TR], b[TC];
#pragma unroll
                for (int u = 0; u < TR; ++u) a[u] = zr[(size_t)kk * ZLD + u * RG];
#pragma unroll
                for (int t = 0; t < TC; ++t) b[t] = xr[(size_t)kk * COLS + t * CG];
#pragma unroll
                for (int u = 0; u < TR; ++u)
#pragma unroll
                    for (int t = 0; t < TC; ++t) cfma(acc[u][t], a[u], b[t]);
            }
        }
    }
    __syncthreads();
    if (worker) {
#pragma unroll
        for (int u = 0; u < TR; ++u) {
            const int row = rg + u * RG;
#pragma unroll
            for (int t = 0; t < TC; ++t) {
                const int col = cg + t * CG;
                if (row < DI * ts && col < M) Gs[(size_t)row * M + col] = acc[u][t];
            }
        }
    }
    __syncthreads();
    terms_epilogue(P, O, Gs, DI, i0, N, T, xc, coff, zadd, alpha, beta, singular, y, tid, nthr);
}

// ---- stored tables -------------------------------------------------------------------------
// For repeated applications (GMRES) the tables of all ordered pairs are built once and kept in
// HBM, laid out for the FP64 tensor-core product: per block of DI destinations (RO row octets
// of 8 table rows, rows il * tsize + idx) and per chunk of 16 sources, a contiguous 2 KB slab
// per row octet and group of 4 sources in the m8n8k4 A-fragment order (lane = 4 * row % 8 +
// source % 4). The inputs are packed per call in the B-fragment order (lane = 4 * column % 8 +
// source % 4), so every fragment load of a warp reads 512 contiguous bytes.
constexpr int SRC_CHUNK = 16;  // sources per stored chunk
constexpr int AS_STAGES = 3;   // cp.async ring of the stored product

__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int K>
__device__ __forceinline__ void cp_async_wait() {
    asm volatile("cp.async.wait_group %0;" ::"n"(K) : "memory");
}
// c += a b on one 8 x 8 FP64 tile (m8n8k4, A row-major, B column-major)
__device__ __forceinline__ void dmma(double (&c)[2], double a, double b) {
    asm("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};"
        : "+d"(c[0]), "+d"(c[1])
        : "d"(a), "d"(b));
}

// CTA = one block of DI destinations x a range of source chunks: builds the chunk tables
// (degrees <= order) exactly as the on-the-fly product does and writes them out in the stored
// order.
__global__ void __launch_bounds__(256) table_store_kernel(DevPlan P, int order, int N, double k,
                                                          const double* __restrict__ pos, int DI, int KJ, int RO,
                                                          int NC, int span, cplx* __restrict__ Z) {
    extern __shared__ __align__(16) unsigned char ts_smem[];
    const int ord1 = order + 1, ts = ord1 * ord1, rows = DI * ts;
    const int ZLD = RO * 8 + 1, npair = DI * KJ;
    cplx* Zs = reinterpret_cast<cplx*>(ts_smem);                          // KJ x ZLD
    cplx* Rs = Zs + (size_t)KJ * ZLD;                                     // npair x (order + 1)
    double4* Ds = reinterpret_cast<double4*>(Rs + (size_t)npair * ord1);  // direction, state
    const int tid = threadIdx.x, nthr = blockDim.x;
    const int i0 = blockIdx.x * DI;
    for (int t = tid; t < KJ * ZLD; t += nthr) Zs[t] = mk(0.0, 0.0);  // padding rows stay zero
    const int jbeg = blockIdx.y * span, jend = min(N, jbeg + span);
    cplx* Zb = Z + (size_t)blockIdx.x * NC * RO * 128;
    for (int j0 = jbeg; j0 < jend; j0 += KJ) {
        __syncthreads();  // the previous chunk is written out
        build_chunk(P, order, N, k, pos, true, i0, j0, DI, KJ, ZLD, Zs, Rs, Ds, tid, nthr);
        __syncthreads();
        // out: per 16-source chunk c, group q of 4 sources, row octet o, lane
        const int total = (KJ / SRC_CHUNK) * 4 * RO * 32;
        for (int it = tid; it < total; it += nthr) {
            const int lane = it & 31, w = it >> 5, o = w % RO, qc = w / RO;
            const int row = o * 8 + (lane >> 2), kk = qc * 4 + (lane & 3);  // qc = 4 c + q
            const cplx v = row < rows ? Zs[(size_t)kk * ZLD + row] : mk(0.0, 0.0);
            const size_t slab = (size_t)(j0 / SRC_CHUNK) * 4 + qc;  // chunk * 4 + q
            Zb[(slab * RO + o) * 32 + lane] = v;
        }
    }
}

// Inputs of ncol columns in the B-fragment order: per chunk, group q, column octet c, lane.
__global__ void pack_sources_kernel(const cplx* __restrict__ x, size_t ldx, int ldin, int N, int M, int NC, int CT,
                                    cplx* __restrict__ Xf) {
    const size_t per = (size_t)NC * 4 * CT * 32;
    const cplx* xc = x + (size_t)blockIdx.y * ldx;
    cplx* out = Xf + (size_t)blockIdx.y * per;
    for (size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x; t < per; t += (size_t)gridDim.x * blockDim.x) {
        const int lane = (int)(t & 31);
        const size_t w = t >> 5;
        const int c = (int)(w % CT);
        const size_t g = w / CT;  // chunk * 4 + q
        const size_t j = g * 4 + (lane & 3);
        const int col = c * 8 + (lane >> 2);
        out[t] = (j < (size_t)N && col < M) ? xc[j * ldin + col] : mk(0.0, 0.0);
    }
}

// y = zadd + alpha x + beta T C x (or the sub-operator O) from the stored tables: CTA = DI
// destinations x one column, a warp per RPW row octets with CT column octets (complex
// accumulators as re and im 8 x 8 FP64 tiles, four m8n8k4 products per complex step:
// re += a.re b.re + a.im (-b.im), im += a.re b.im + a.im b.re, each B fragment used for RPW
// row octets); chunks of 16 sources through a 3-stage cp.async ring; then the term lists.
template <int CT, int RPW>
__global__ void __launch_bounds__(256, 1)
    apply_stored_kernel(DevPlan P, SubOp O, int N, const cplx* __restrict__ Z, const cplx* __restrict__ Xf, int NC,
                        int DI, int RO, const cplx* __restrict__ T, const cplx* __restrict__ x, size_t ldx,
                        const cplx* __restrict__ zadd, double alpha, double beta, cplx* __restrict__ y) {
    extern __shared__ __align__(16) unsigned char as_smem[];
    const int tid = threadIdx.x, nthr = blockDim.x, lane = tid & 31, o0 = (tid >> 5) * RPW;
    const int ABLK = RO * 128, BBLK = CT * 128, SBLK = ABLK + BBLK;  // complex entries per chunk
    cplx* ring = reinterpret_cast<cplx*>(as_smem);
    const cplx* Zb = Z + (size_t)blockIdx.x * NC * ABLK;
    const cplx* Xb = Xf + (size_t)blockIdx.y * NC * BBLK;
    auto load = [&](int stage, int kc) {
        cplx* dst = ring + (size_t)stage * SBLK;
        const cplx* sa = Zb + (size_t)kc * ABLK;
        const cplx* sb = Xb + (size_t)kc * BBLK;
        for (int t = tid; t < SBLK; t += nthr) cp_async16(dst + t, t < ABLK ? sa + t : sb + (t - ABLK));
    };
    double re[RPW][CT][2], im[RPW][CT][2];
#pragma unroll
    for (int r = 0; r < RPW; ++r)
#pragma unroll
        for (int c = 0; c < CT; ++c) re[r][c][0] = re[r][c][1] = im[r][c][0] = im[r][c][1] = 0.0;
    // row octets past RO (the last warp of an odd count) skip their products, warp-uniformly
    const int nr = min(RPW, RO - o0);
#pragma unroll
    for (int s = 0; s < AS_STAGES - 1; ++s) {
        if (s < NC) load(s, s);
        cp_async_commit();
    }
    for (int kc = 0; kc < NC; ++kc) {
        cp_async_wait<AS_STAGES - 2>();
        __syncthreads();  // chunk kc landed for every thread; the stage of chunk kc - 1 is free
        if (kc + AS_STAGES - 1 < NC) load((kc + AS_STAGES - 1) % AS_STAGES, kc + AS_STAGES - 1);
        cp_async_commit();
        const cplx* As = ring + (size_t)(kc % AS_STAGES) * SBLK;
        const cplx* Bs = As + ABLK;
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            cplx a[RPW];
#pragma unroll
            for (int r = 0; r < RPW; ++r) a[r] = r < nr ? As[(q * RO + o0 + r) * 32 + lane] : mk(0.0, 0.0);
#pragma unroll
            for (int c = 0; c < CT; ++c) {
                const cplx b = Bs[(q * CT + c) * 32 + lane];
#pragma unroll
                for (int r = 0; r < RPW; ++r) {
                    if (r < nr) {
                        dmma(re[r][c], a[r].x, b.x);
                        dmma(re[r][c], a[r].y, -b.y);
                        dmma(im[r][c], a[r].x, b.y);
                        dmma(im[r][c], a[r].y, b.x);
                    }
                }
            }
        }
    }
    cp_async_wait<0>();
    __syncthreads();  // the ring is free for G
    cplx* Gs = reinterpret_cast<cplx*>(as_smem);
    const int M = 2 * O.nsrc, rows = DI * (O.order + 1) * (O.order + 1);
#pragma unroll
    for (int r = 0; r < RPW; ++r) {
        const int row = (o0 + r) * 8 + (lane >> 2);
        if (row < rows) {
#pragma unroll
            for (int c = 0; c < CT; ++c) {
                const int col = c * 8 + 2 * (lane & 3);
                if (col < M) {
                    Gs[(size_t)row * M + col] = mk(re[r][c][0], im[r][c][0]);
                    Gs[(size_t)row * M + col + 1] = mk(re[r][c][1], im[r][c][1]);
                }
            }
        }
    }
    __syncthreads();
    const size_t coff = (size_t)blockIdx.y * ldx;
    terms_epilogue(P, O, Gs, DI, blockIdx.x * DI, N, T, x + coff, coff, zadd, alpha, beta, true, y, tid, nthr);
}

// ---- bulk-copy pipeline of the stored product ---------------------------------------------
constexpr int AT_STAGES = AS_STAGES;  // ring depth of the bulk-copy pipeline (2 CTAs per SM at lmax <= 4)

__device__ __forceinline__ uint32_t as_smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }
__device__ __forceinline__ void as_mbar_init(uint32_t bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}
__device__ __forceinline__ void as_mbar_expect_tx(uint32_t bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}
__device__ __forceinline__ void as_mbar_arrive(uint32_t bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}
__device__ __forceinline__ bool as_mbar_try(uint32_t bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(bar), "r"(parity)
        : "memory");
    return ok != 0;
}
// Bounded wait on a phase: false after 2 s (recorded in abort_flag) or once another warp gave up.
__device__ __forceinline__ bool as_mbar_wait(uint32_t bar, uint32_t parity, volatile int* abort_flag) {
    if (as_mbar_try(bar, parity)) return true;
    unsigned long long t0;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t0));
    for (unsigned it = 1;; ++it) {
        if (as_mbar_try(bar, parity)) return true;
        if ((it & 63u) == 0) {
            if (*abort_flag) return false;
            unsigned long long t;
            asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
            if (t - t0 > 2000000000ull) {
                *abort_flag = 1;
                return false;
            }
        }
    }
}
// contiguous global -> shared copy completing on an mbarrier (16-byte aligned, size % 16 == 0)
__device__ __forceinline__ void as_bulk_load(uint32_t dst, const void* src, uint32_t bytes, uint32_t bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
        "l"(src), "r"(bytes), "r"(bar)
        : "memory");
}

// The stored product with a producer warp: lane 0 of the last warp streams the 16-source chunks
// (table slab and packed inputs, each one contiguous bulk copy) into a 3-stage ring, each stage
// completing on its full barrier; the product warps take a stage once its full barrier flips
// and release it through its empty barrier (one arrival per warp), so no CTA-wide barrier
// sits in the loop. Every wait is bounded (2 s): on a timeout the kernel records status 8,
// waits (bounded) for the copies in flight and returns without writing y.
template <int CT, int RPW>
__global__ void __launch_bounds__(288, 1)
    apply_stored_tma_kernel(DevPlan P, SubOp O, int N, const cplx* __restrict__ Z, const cplx* __restrict__ Xf,
                            int NC, int DI, int RO, const cplx* __restrict__ T, const cplx* __restrict__ x, size_t ldx,
                            const cplx* __restrict__ zadd, double alpha, double beta, cplx* __restrict__ y,
                            int* __restrict__ status) {
    extern __shared__ __align__(128) unsigned char at_smem[];
    __shared__ __align__(8) uint64_t bars[2 * AT_STAGES];
    __shared__ int s_abort;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int W = (RO + RPW - 1) / RPW;  // product warps; warp W loads
    const int ABLK = RO * 128, BBLK = CT * 128, SBLK = ABLK + BBLK;  // complex entries per chunk
    cplx* ring = reinterpret_cast<cplx*>(at_smem);
    const cplx* Zb = Z + (size_t)blockIdx.x * NC * ABLK;
    const cplx* Xb = Xf + (size_t)blockIdx.y * NC * BBLK;
    const uint32_t full0 = as_smem_u32(bars), empty0 = full0 + 8 * AT_STAGES;
    if (tid == 0) {
        for (int s = 0; s < AT_STAGES; ++s) {
            as_mbar_init(full0 + 8 * s, 1);
            as_mbar_init(empty0 + 8 * s, W);
        }
        s_abort = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    volatile int* abort_flag = &s_abort;
    double re[RPW][CT][2], im[RPW][CT][2];
#pragma unroll
    for (int r = 0; r < RPW; ++r)
#pragma unroll
        for (int c = 0; c < CT; ++c) re[r][c][0] = re[r][c][1] = im[r][c][0] = im[r][c][1] = 0.0;
    const int o0 = warp * RPW;
    if (warp == W) {
        if (lane == 0) {
            int kc = 0;
            for (; kc < NC; ++kc) {
                const int s = kc % AT_STAGES;
                if (!as_mbar_wait(empty0 + 8 * s, ((kc / AT_STAGES) & 1) ^ 1, abort_flag)) break;
                const uint32_t dst = as_smem_u32(ring + (size_t)s * SBLK);
                as_mbar_expect_tx(full0 + 8 * s, (uint32_t)SBLK * 16u);
                as_bulk_load(dst, Zb + (size_t)kc * ABLK, (uint32_t)ABLK * 16u, full0 + 8 * s);
                as_bulk_load(dst + (uint32_t)ABLK * 16u, Xb + (size_t)kc * BBLK, (uint32_t)BBLK * 16u, full0 + 8 * s);
            }
            if (*abort_flag) {
                // drain: the last load issued into every stage lands before the CTA exits
                volatile int never = 0;
                for (int s = 0; s < AT_STAGES; ++s) {
                    const int last = kc - 1 - ((kc - 1 - s) % AT_STAGES + AT_STAGES) % AT_STAGES;
                    if (last >= 0) as_mbar_wait(full0 + 8 * s, (last / AT_STAGES) & 1, &never);
                }
            }
        }
    } else if (warp < W) {
        const int nr = min(RPW, RO - o0);
        for (int kc = 0; kc < NC; ++kc) {
            const int s = kc % AT_STAGES;
            if (!as_mbar_wait(full0 + 8 * s, (kc / AT_STAGES) & 1, abort_flag)) break;
            const cplx* As = ring + (size_t)s * SBLK;
            const cplx* Bs = As + ABLK;
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                cplx a[RPW];
#pragma unroll
                for (int r = 0; r < RPW; ++r) a[r] = r < nr ? As[(q * RO + o0 + r) * 32 + lane] : mk(0.0, 0.0);
#pragma unroll
                for (int c = 0; c < CT; ++c) {
                    const cplx b = Bs[(q * CT + c) * 32 + lane];
#pragma unroll
                    for (int r = 0; r < RPW; ++r) {
                        if (r < nr) {
                            dmma(re[r][c], a[r].x, b.x);
                            dmma(re[r][c], a[r].y, -b.y);
                            dmma(im[r][c], a[r].x, b.y);
                            dmma(im[r][c], a[r].y, b.x);
                        }
                    }
                }
            }
            __syncwarp();
            if (lane == 0) as_mbar_arrive(empty0 + 8 * s);
        }
    }
    __syncthreads();  // every chunk consumed: no copy in flight, the ring is free for G
    if (s_abort) {
        if (tid == 0 && status) atomicExch(status, 8);
        return;
    }
    cplx* Gs = reinterpret_cast<cplx*>(at_smem);
    const int M = 2 * O.nsrc, rows = DI * (O.order + 1) * (O.order + 1);
    if (warp < W) {
#pragma unroll
        for (int r = 0; r < RPW; ++r) {
            const int row = (o0 + r) * 8 + (lane >> 2);
            if (row < rows) {
#pragma unroll
                for (int c = 0; c < CT; ++c) {
                    const int col = c * 8 + 2 * (lane & 3);
                    if (col < M) {
                        Gs[(size_t)row * M + col] = mk(re[r][c][0], im[r][c][0]);
                        Gs[(size_t)row * M + col + 1] = mk(re[r][c][1], im[r][c][1]);
                    }
                }
            }
        }
    }
    __syncthreads();
    const size_t coff = (size_t)blockIdx.y * ldx;
    terms_epilogue(P, O, Gs, DI, blockIdx.x * DI, N, T, x + coff, coff, zadd, alpha, beta, true, y, tid,
                   blockDim.x);
}

}  // namespace

bool stored_tables_enabled() {
    const char* e = getenv("TCU_APPLY");
    return !(e && (strcmp(e, "fly") == 0 || strcmp(e, "terms") == 0));
}

bool apply_gemm_supported(const DevPlan& P) {
    if (P.L < 2 || P.L > 5) return false;
    const char* e = getenv("TCU_APPLY");  // "terms": the per-pair term-sum kernels instead
    return !(e && strcmp(e, "terms") == 0);
}

template <int TR, int TC>
static void launch_shape(const DevPlan& P, const SubOp& O, const GemmShape& s, int N, double k, const double* pos,
                         const cplx* T, const cplx* x, size_t ldx, int ncol, const cplx* zadd, double alpha,
                         double beta, bool singular, cplx* y, cudaStream_t st) {
    const dim3 grid((unsigned)((N + s.DI - 1) / s.DI), (unsigned)ncol);
    apply_gemm_kernel<TR, TC><<<grid, s.RG * s.CG, gemm_smem(O, s), st>>>(P, O, N, k, pos, T, x, ldx, zadd, alpha,
                                                                          beta, singular, y, s.DI, s.RG, s.CG, s.KJ);
}

void launch_apply_gemm(const DevPlan& P, int N, double k, const double* pos, const cplx* T, const cplx* x, size_t ldx,
                       int ncol, const cplx* zadd, double alpha, double beta, bool singular, cplx* y,
                       cudaStream_t st) {
    if (N <= 0 || ncol <= 0) return;
    const GemmShape s = gemm_shape(P.L);
    const SubOp O{P.nlm, P.nlm, P.order, 2 * P.nlm, 2 * P.nlm};
    switch (P.L) {
        case 2: launch_shape<4, 2>(P, O, s, N, k, pos, T, x, ldx, ncol, zadd, alpha, beta, singular, y, st); break;
        case 3: launch_shape<4, 3>(P, O, s, N, k, pos, T, x, ldx, ncol, zadd, alpha, beta, singular, y, st); break;
        case 4: launch_shape<4, 4>(P, O, s, N, k, pos, T, x, ldx, ncol, zadd, alpha, beta, singular, y, st); break;
        default: launch_shape<4, 5>(P, O, s, N, k, pos, T, x, ldx, ncol, zadd, alpha, beta, singular, y, st); break;
    }
}

void launch_apply_dipole(const DevPlan& P, int N, double k, const double* pos, const cplx* T, const cplx* z,
                         bool dipole_rows, const cplx* zadd, double alpha, double beta, cplx* y, cudaStream_t st) {
    if (N <= 0) return;
    StageScope sc(ST_COARSE, st);
    const int ndst = dipole_rows ? 3 : P.nlm;
    const SubOp O{3, ndst, 1 + (dipole_rows ? 1 : P.L), 6, 2 * ndst};
    const GemmShape s = sub_shape((O.order + 1) * (O.order + 1));
    launch_shape<4, 2>(P, O, s, N, k, pos, T, z, 0, 1, zadd, alpha, beta, true, y, st);
}

// ---- stored tables: host side ----------------------------------------------------------------
namespace {
SubOp stored_subop(const DevPlan& P, int kind) {
    switch (kind) {
        case STORED_DIPOLE_SOURCES: return {3, P.nlm, 1 + P.L, 6, 2 * P.nlm};
        case STORED_DIPOLE_BLOCK: return {3, 3, 2, 6, 6};
        default: return {P.nlm, P.nlm, P.order, 2 * P.nlm, 2 * P.nlm};
    }
}
// full operator: lmax 2..5; dipole blocks: tables of at most 128 entries (one destination per
// block then fills at most 16 row octets, the 8 warps of the product)
bool stored_kind_ok(const DevPlan& P, int kind) {
    if (kind == STORED_FULL) return P.L >= 2 && P.L <= 5;
    if (kind != STORED_DIPOLE_SOURCES && kind != STORED_DIPOLE_BLOCK) return false;
    const int order = stored_subop(P, kind).order;
    return (order + 1) * (order + 1) <= 128;
}
struct StoredLayout {
    SubOp O;
    int DI, KJ, RO, CT, NC, nblk, RPW;  // RPW: row octets per warp of the product
    size_t z_elems, xf_per_col;
};
StoredLayout stored_layout(const DevPlan& P, int N, int kind) {
    StoredLayout l;
    l.O = stored_subop(P, kind);
    const int ts = (l.O.order + 1) * (l.O.order + 1);
    l.DI = std::max(1, 128 / ts);  // about 128 table rows per destination block
    l.KJ = 32;
    l.RO = (l.DI * ts + 7) / 8;
    l.CT = (2 * l.O.nsrc + 7) / 8;
    l.RPW = 2;
    l.NC = (N + l.KJ - 1) / l.KJ * (l.KJ / SRC_CHUNK);
    l.nblk = (N + l.DI - 1) / l.DI;
    l.z_elems = (size_t)l.nblk * l.NC * l.RO * 128;
    l.xf_per_col = (size_t)l.NC * l.CT * 128;
    return l;
}
size_t stored_smem(const StoredLayout& l) {
    const size_t ring = (size_t)AS_STAGES * (l.RO + l.CT) * 128 * sizeof(cplx);
    const size_t g = (size_t)l.DI * (l.O.order + 1) * (l.O.order + 1) * 2 * l.O.nsrc * sizeof(cplx);
    return ring > g ? ring : g;
}
size_t store_smem(const StoredLayout& l) {
    const size_t npair = (size_t)l.DI * l.KJ;
    return ((size_t)l.KJ * (l.RO * 8 + 1) + npair * (l.O.order + 1)) * sizeof(cplx) + npair * sizeof(double4);
}
}  // namespace

size_t stored_tables_bytes(const DevPlan& P, int N, int kind) {
    if (!stored_kind_ok(P, kind) || N <= 0) return 0;
    return stored_layout(P, N, kind).z_elems * sizeof(cplx);
}

size_t stored_inputs_bytes(const DevPlan& P, int N, int kind, int ncol) {
    if (!stored_kind_ok(P, kind) || N <= 0) return 0;
    return stored_layout(P, N, kind).xf_per_col * (size_t)ncol * sizeof(cplx);
}

void build_stored_tables(const DevPlan& P, int N, double k, const double* pos, int kind, cplx* Z, cudaStream_t st) {
    if (N <= 0 || !stored_kind_ok(P, kind)) return;
    StageScope sc(kind == STORED_FULL ? ST_APPLY : ST_COARSE, st);
    const StoredLayout l = stored_layout(P, N, kind);
    const int nchunk = (N + l.KJ - 1) / l.KJ;
    const int ysplit = std::min(nchunk, std::max(1, (4 * 148 + l.nblk - 1) / l.nblk));
    const int span = (nchunk + ysplit - 1) / ysplit * l.KJ;
    const dim3 grid((unsigned)l.nblk, (unsigned)((nchunk * l.KJ + span - 1) / span));
    table_store_kernel<<<grid, 256, store_smem(l), st>>>(P, l.O.order, N, k, pos, l.DI, l.KJ, l.RO, l.NC, span, Z);
}

void launch_apply_stored(const DevPlan& P, int N, int kind, const cplx* Z, const cplx* T, const cplx* x, size_t ldx,
                         int ncol, const cplx* zadd, double alpha, double beta, cplx* y, cplx* Xf, int* status,
                         cudaStream_t st) {
    if (N <= 0 || ncol <= 0 || !stored_kind_ok(P, kind)) return;
    StageScope sc(kind == STORED_FULL ? ST_APPLY : ST_COARSE, st);
    const StoredLayout l = stored_layout(P, N, kind);
    const int M = 2 * l.O.nsrc;
    const dim3 pgrid((unsigned)std::min<size_t>((l.xf_per_col + 255) / 256, 1024), (unsigned)ncol);
    pack_sources_kernel<<<pgrid, 256, 0, st>>>(x, ldx, l.O.ldin, N, M, l.NC, l.CT, Xf);
    const dim3 grid((unsigned)l.nblk, (unsigned)ncol);
    const size_t smem = stored_smem(l);
    const int threads = (l.RO + l.RPW - 1) / l.RPW * 32;
    // bulk-copy pipeline, except at 6 column octets (lmax 4) where the cp.async ring measured
    // faster (1.43 against 1.58 ms at 1024 spheres); TCU_STORED_PIPE=cpasync or tma forces one
    const char* pipe = getenv("TCU_STORED_PIPE");
    const bool cpasync = pipe ? strcmp(pipe, "cpasync") == 0 : l.CT == 6;
#define TCU_STORED(CT, RPW)                                                                                       \
    if (cpasync)                                                                                                  \
        apply_stored_kernel<CT, RPW><<<grid, threads, smem, st>>>(P, l.O, N, Z, Xf, l.NC, l.DI, l.RO, T, x, ldx,   \
                                                                 zadd, alpha, beta, y);                            \
    else                                                                                                          \
        apply_stored_tma_kernel<CT, RPW><<<grid, threads + 32, smem, st>>>(P, l.O, N, Z, Xf, l.NC, l.DI, l.RO, T, \
                                                                          x, ldx, zadd, alpha, beta, y, status)
    switch (l.CT) {
        case 1: TCU_STORED(1, 2); break;
        case 2: TCU_STORED(2, 2); break;
        case 4: TCU_STORED(4, 2); break;
        case 6: TCU_STORED(6, 2); break;
        default: TCU_STORED(9, 2); break;
    }
#undef TCU_STORED
}

void apply_gemm_init_attributes() {
    cudaFuncSetAttribute(apply_gemm_kernel<4, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
    cudaFuncSetAttribute(apply_gemm_kernel<4, 3>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
    cudaFuncSetAttribute(apply_gemm_kernel<4, 4>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
    cudaFuncSetAttribute(apply_gemm_kernel<4, 5>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
    cudaFuncSetAttribute(table_store_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
    cudaFuncSetAttribute(apply_stored_kernel<1, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
    cudaFuncSetAttribute(apply_stored_tma_kernel<1, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
    cudaFuncSetAttribute(apply_stored_kernel<2, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
    cudaFuncSetAttribute(apply_stored_tma_kernel<2, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
    cudaFuncSetAttribute(apply_stored_kernel<4, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
    cudaFuncSetAttribute(apply_stored_tma_kernel<4, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
    cudaFuncSetAttribute(apply_stored_kernel<6, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
    cudaFuncSetAttribute(apply_stored_tma_kernel<6, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
    cudaFuncSetAttribute(apply_stored_kernel<9, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
    cudaFuncSetAttribute(apply_stored_tma_kernel<9, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
}

}  // namespace tcu
