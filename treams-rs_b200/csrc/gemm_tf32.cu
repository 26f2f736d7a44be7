// Trailing update of the mixed-precision LU on the 5th-generation tensor cores:
//   A22 -= L21 U12   (complex64, column-major, in place)
// as one real GEMM D = Lemb * U^T with
//   Lemb[2mu+c][2k+c'] = { Re L, -Im L ; Im L, Re L }   (2m x 2w, K-major)
//   U[nu][2k+c']       = interleaved (Re, Im) of column nu of U12   (n' x 2w, K-major)
// so that D[2mu+c][nu] is part c of (L21 U12)[mu][nu] and the 2m x n' result maps onto
// the interleaved storage of A22 (real leading dimension 2n).
//
// Precision: every operand is split x = hi + lo into two 11-bit-significand pieces and the
// passes accumulate in FP32 in TMEM: by default two, hi*hi + lo*hi (the B operand rounded to
// TF32, about 2^-11 relative per term; the FP64 refinement takes one sweep more), with
// TCU_SPLIT=tf32x3 or f16 three, hi*hi + hi*lo + lo*hi (the lo*lo term is below FP32
// rounding). Two piece formats:
//   FP16 (TCU_SPLIT=f16): each row of each operand (a complex row of L21, a column of U12) is
//     first scaled by its own power of two 2^(14 - ceil log2 max|row|) (computed in the
//     packing kernels; no host round trip), hi = f16(x s), lo = f16(x s - hi);
//     tcgen05.mma kind::f16 runs at twice the TF32 rate and the epilogue multiplies each
//     accumulator entry by the exact power of two 1/(s_row s_col). Pieces below the FP16
//     normal range only lose absolute accuracy under 2^-38 of their row's maximum.
//   TF32 (default): hi = tf32(x), lo = tf32(x - hi), tcgen05.mma kind::tf32.
// Both give a product accurate to about 2^-22 of max|A| max|B| per term.
//
// Kernel layout (persistent, one CTA per SM, 192 threads):
//   warp 0     TMA producer: 64-byte-swizzled boxes (64-byte K rows) of the four packed
//              operands into a 4-stage shared-memory ring (48 KB per stage), mbarrier complete_tx;
//   warp 1     TMEM allocator and MMA issuer (one thread): 2 K-steps x 2 or 3 passes per stage
//              into a 128 x 256 FP32 accumulator, double-buffered in TMEM (512 columns);
//   warps 2-5  epilogue: tcgen05.ld 32 columns at a time into a shared-memory staging buffer,
//              TMA reduce-add of -D into A22.
// Every mbarrier wait is bounded; on timeout the kernel records status 8, drains its TMA
// loads, frees TMEM and returns.
#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include <cuda_fp16.h>

#include <algorithm>
#include <atomic>
#include <cstdlib>
#include <cstring>

#include "kernels.h"
#include "precond.h"

namespace tcu {

constexpr int TB_M = 128;       // real rows per tile (64 complex rows)
constexpr int TB_N = 256;       // columns per tile
constexpr int TB_K = 16;        // floats per K chunk (one 64-byte swizzle row); 32 for FP16 pieces
constexpr int TB_STAGES = 4;
constexpr int A_BYTES = TB_M * TB_K * 4;   // 8 KB
constexpr int B_BYTES = TB_N * TB_K * 4;   // 16 KB
constexpr int STAGE_BYTES = 2 * A_BYTES + 2 * B_BYTES;  // 48 KB
constexpr int TMEM_COLS = 2 * TB_N;        // two accumulators
constexpr int EPI_COLS = 32;                         // columns per epilogue staging buffer
constexpr int EPI_BYTES = TB_M * EPI_COLS * 4;         // 16 KB
constexpr size_t TF32_SMEM = (size_t)TB_STAGES * STAGE_BYTES + 2 * EPI_BYTES + 1024 + 256;

// ---- device helpers ---------------------------------------------------------------------
__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ unsigned long long gtimer() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint32_t bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}
__device__ __forceinline__ bool mbar_try(uint32_t bar, uint32_t parity) {
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
// Bounded wait: false after 2 s or when another role has aborted.
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity, volatile int* abort_flag) {
    if (mbar_try(bar, parity)) return true;
    unsigned long long t0 = gtimer();
    for (unsigned it = 1;; ++it) {
        if (mbar_try(bar, parity)) return true;
        if ((it & 63u) == 0) {
            if (*abort_flag) return false;
            if (gtimer() - t0 > 2000000000ull) {
                *abort_flag = 1;
                return false;
            }
        }
    }
}

__device__ __forceinline__ void tma_load_2d(uint32_t dst, const CUtensorMap* map, int x, int y, uint32_t bar) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], "
        "[%4];" ::"r"(dst),
        "l"((uint64_t)map), "r"(x), "r"(y), "r"(bar)
        : "memory");
}

// K-major, 64-byte swizzled operand tile: rows of 16 floats, 8-row groups 512 bytes apart.
__device__ __forceinline__ uint64_t swz_desc(uint32_t addr) {
    uint64_t d = 0;
    d |= (uint64_t)((addr >> 4) & 0x3FFFu);
    d |= (uint64_t)1 << 16;             // leading byte offset (unused for swizzled K-major)
    d |= (uint64_t)(512 >> 4) << 32;    // stride byte offset: next 8-row group
    d |= (uint64_t)1 << 46;             // descriptor version (sm_100)
    d |= (uint64_t)4 << 61;             // SWIZZLE_64B
    return d;
}

// Tile t of the persistent loop: groups of 16 M-tiles sweep all N-tiles, so the CTAs in
// flight share a few A and B tiles in L2.
constexpr int TILE_GROUP = 16;
__device__ __forceinline__ void tile_coords(int t, int tiles_m, int tiles_n, int& tm, int& tn) {
    int per_group = TILE_GROUP * tiles_n;
    int g = t / per_group;
    int first = g * TILE_GROUP;
    int gm = min(TILE_GROUP, tiles_m - first);
    int local = t - g * per_group;
    tm = first + local % gm;
    tn = local / gm;
}

__device__ __forceinline__ void mma_tf32(uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t idesc, uint32_t acc) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}" ::"r"(d_tmem),
        "l"(a), "l"(b), "r"(idesc), "r"(acc)
        : "memory");
}
__device__ __forceinline__ void mma_f16(uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t idesc, uint32_t acc) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(d_tmem),
        "l"(a), "l"(b), "r"(idesc), "r"(acc)
        : "memory");
}
template <bool F16>
__device__ __forceinline__ void mma_split(uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t idesc, uint32_t acc) {
    if (F16)
        mma_f16(d_tmem, a, b, idesc, acc);
    else
        mma_tf32(d_tmem, a, b, idesc, acc);
}
// Power-of-two scale that maps max |x| to (2^13, 2^14]: exact, and far inside the FP16 range.
__device__ __forceinline__ float f16_scale(float mx) {
    if (!(mx > 0.0f) || !isfinite(mx)) return 1.0f;
    int e;
    frexpf(mx, &e);  // mx = f 2^e, 0.5 <= f < 1
    return ldexpf(1.0f, 14 - e);
}
__device__ __forceinline__ void mma_commit(uint32_t bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar) : "memory");
}
__device__ __forceinline__ void fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }

__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float* v) {
    uint32_t r[32];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
        "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
          "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
          "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 32; ++i) v[i] = __uint_as_float(r[i]);
}

// ---- the GEMM ---------------------------------------------------------------------------
struct Tf32Args {
    float* C;        // A viewed as floats
    size_t ldc;      // 2n (floats per column)
    int row0;        // 2 r0: first real row of A22
    int col0;        // r0
    int m2;          // real rows of A22 (2m)
    int ncols;       // columns of A22
    int kchunks;     // K / TB_K
    int tiles_m, tiles_n, tiles;
    int* status;
    const float* sA;      // FP16 pieces: scale of each complex row of the A operand (m2 / 2), else null
    const float* sB;      // FP16 pieces: scale of each row of the B operand (ncols)
};

template <bool F16, bool TWO>
__global__ void __launch_bounds__(192, 1) tf32_update_kernel(const __grid_constant__ CUtensorMap mAhi,
                                                             const __grid_constant__ CUtensorMap mAlo,
                                                             const __grid_constant__ CUtensorMap mBhi,
                                                             const __grid_constant__ CUtensorMap mBlo,
                                                             const __grid_constant__ CUtensorMap mC, Tf32Args args) {
    extern __shared__ uint8_t smem_raw[];
    uint32_t base = smem_u32(smem_raw);
    uint32_t tiles_smem = (base + 1023u) & ~1023u;  // 1024-byte aligned stage ring
    const uint32_t epi_smem = tiles_smem + TB_STAGES * STAGE_BYTES;  // 2 staging buffers
    float* epi = (float*)(smem_raw + (epi_smem - base));
    uint8_t* ctrl = smem_raw + (tiles_smem - base) + TB_STAGES * STAGE_BYTES + 2 * EPI_BYTES;
    // barriers: full[S], empty[S], tmem_full[2], tmem_empty[2]
    uint64_t* bars = (uint64_t*)ctrl;
    uint32_t* tmem_slot = (uint32_t*)(ctrl + 8 * (2 * TB_STAGES + 4));
    volatile int* abort_flag = (volatile int*)(tmem_slot + 1);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    auto bar = [&](int i) { return smem_u32(&bars[i]); };
    constexpr int EMPTY = TB_STAGES, TFULL = 2 * TB_STAGES, TEMPTY = 2 * TB_STAGES + 2;
    if (threadIdx.x == 0) {
        for (int s = 0; s < TB_STAGES; ++s) {
            mbar_init(bar(s), 1);
            mbar_init(bar(EMPTY + s), 1);
        }
        for (int a = 0; a < 2; ++a) {
            mbar_init(bar(TFULL + a), 1);
            mbar_init(bar(TEMPTY + a), 128);
        }
        *abort_flag = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 1) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                     "r"(TMEM_COLS));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    __syncthreads();
    fence_after();
    const uint32_t tmem_base = *tmem_slot;

    if (warp == 0) {
        if (lane == 0) {
            int step = 0;
            for (int t = blockIdx.x; t < args.tiles && !*abort_flag; t += gridDim.x) {
                int tm, tn;
                tile_coords(t, args.tiles_m, args.tiles_n, tm, tn);
                for (int kb = 0; kb < args.kchunks; ++kb, ++step) {
                    int s = step % TB_STAGES;
                    uint32_t ph = (step / TB_STAGES) & 1;
                    if (!mbar_wait(bar(EMPTY + s), ph ^ 1, abort_flag)) break;
                    uint32_t st = tiles_smem + s * STAGE_BYTES;
                    mbar_expect_tx(bar(s), TWO ? STAGE_BYTES - B_BYTES : STAGE_BYTES);
                    tma_load_2d(st, &mAhi, kb * TB_K, tm * TB_M, bar(s));
                    tma_load_2d(st + A_BYTES, &mAlo, kb * TB_K, tm * TB_M, bar(s));
                    tma_load_2d(st + 2 * A_BYTES, &mBhi, kb * TB_K, tn * TB_N, bar(s));
                    if (!TWO) tma_load_2d(st + 2 * A_BYTES + B_BYTES, &mBlo, kb * TB_K, tn * TB_N, bar(s));
                }
            }
            if (*abort_flag) {
                // drain: wait (bounded) for the loads of every stage still in flight
                volatile int never = 0;
                for (int s = 0; s < TB_STAGES; ++s) {
                    int last = step - 1 - ((step - 1 - s) % TB_STAGES + TB_STAGES) % TB_STAGES;
                    if (last >= 0) mbar_wait(bar(s), (last / TB_STAGES) & 1, &never);
                }
            }
        }
    } else if (warp == 1) {
        if (lane == 0) {
            // D F32; A, B TF32 (2) or F16 (0); K-major; N >> 3 at bit 17, M >> 4 at bit 24
            const uint32_t ab = F16 ? 0u : 2u;
            const uint32_t idesc = (1u << 4) | (ab << 7) | (ab << 10) | ((uint32_t)(TB_N >> 3) << 17) |
                                   ((uint32_t)(TB_M >> 4) << 24);
            int step = 0, it = 0;
            for (int t = blockIdx.x; t < args.tiles && !*abort_flag; t += gridDim.x, ++it) {
                int acc = it & 1;
                uint32_t aph = (it >> 1) & 1;
                if (!mbar_wait(bar(TEMPTY + acc), aph ^ 1, abort_flag)) break;
                fence_after();
                uint32_t d = tmem_base + (uint32_t)(acc * TB_N);
                bool ok = true;
                for (int kb = 0; kb < args.kchunks; ++kb, ++step) {
                    int s = step % TB_STAGES;
                    uint32_t ph = (step / TB_STAGES) & 1;
                    if (!mbar_wait(bar(s), ph, abort_flag)) {
                        ok = false;
                        break;
                    }
                    fence_after();
                    uint32_t st = tiles_smem + s * STAGE_BYTES;
#pragma unroll
                    for (int ks = 0; ks < 2; ++ks) {  // two 32-byte K-steps per 64-byte row
                        uint64_t ahi = swz_desc(st + ks * 32), alo = swz_desc(st + A_BYTES + ks * 32);
                        uint64_t bhi = swz_desc(st + 2 * A_BYTES + ks * 32);
                        uint64_t blo = swz_desc(st + 2 * A_BYTES + B_BYTES + ks * 32);
                        uint32_t first = (kb == 0 && ks == 0) ? 0u : 1u;
                        mma_split<F16>(d, ahi, bhi, idesc, first);
                        if (!TWO) mma_split<F16>(d, ahi, blo, idesc, 1u);
                        mma_split<F16>(d, alo, bhi, idesc, 1u);
                    }
                    mma_commit(bar(EMPTY + s));
                }
                if (!ok) break;
                mma_commit(bar(TFULL + acc));
            }
        }
    } else {
        // Epilogue: -D goes through a shared-memory staging buffer ([64 columns][128 rows])
        // and a TMA reduce-add into A22 in L2, so no thread waits on a load of A22.
        const int q = warp & 3;  // TMEM lane quarter of this warp
        const int R = q * 32 + lane;
        const bool issuer = (warp == 2 && lane == 0);
        volatile int* s_go = abort_flag + 1;  // the issuer's wait result, shared by the 4 warps
        // FP16 pieces: -1 / (row scale x column scale) undoes the operand scaling exactly
        const int grow = R;  // row of the tile this thread stores
        int it = 0, e = 0;
        for (int t = blockIdx.x; t < args.tiles; t += gridDim.x, ++it) {
            int acc = it & 1;
            uint32_t aph = (it >> 1) & 1;
            // one thread waits (bounded) and the four warps take its decision together, so a
            // time-out cannot leave some of them at the named barrier
            if (issuer) *s_go = (!*abort_flag && mbar_wait(bar(TFULL + acc), aph, abort_flag)) ? 1 : 0;
            asm volatile("bar.sync 1, 128;" ::: "memory");
            if (!*s_go) break;
            fence_after();
            int tm, tn;
            tile_coords(t, args.tiles_m, args.tiles_n, tm, tn);
            float rowneg = -1.0f;
            if (F16) {
                const int mu = (tm * TB_M + grow) >> 1;
                rowneg = mu < (args.m2 >> 1) ? -1.0f / __ldg(&args.sA[mu]) : -1.0f;
            }
            for (int sub = 0; sub < TB_N / EPI_COLS; ++sub, ++e) {
                const int buf = e & 1;
                if (issuer) asm volatile("cp.async.bulk.wait_group.read 1;" ::: "memory");
                asm volatile("bar.sync 1, 128;" ::: "memory");
                float* stage = epi + buf * (TB_M * EPI_COLS);
#pragma unroll
                for (int cb = 0; cb < EPI_COLS / 32; ++cb) {
                    float v[32];
                    uint32_t taddr = tmem_base + ((uint32_t)(q * 32) << 16) +
                                     (uint32_t)(acc * TB_N + sub * EPI_COLS + cb * 32);
                    tmem_ld32(taddr, v);
#pragma unroll
                    for (int jj = 0; jj < 32; ++jj) {
                        float f = rowneg;
                        if (F16) {
                            const int col = tn * TB_N + sub * EPI_COLS + cb * 32 + jj;
                            f = col < args.ncols ? rowneg / __ldg(&args.sB[col]) : rowneg;
                        }
                        stage[(cb * 32 + jj) * TB_M + R] = f * v[jj];
                    }
                }
                asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
                asm volatile("bar.sync 1, 128;" ::: "memory");
                if (issuer) {
                    int x = args.row0 + tm * TB_M, y = args.col0 + tn * TB_N + sub * EPI_COLS;
                    asm volatile(
                        "cp.reduce.async.bulk.tensor.2d.global.shared::cta.add.tile.bulk_group [%0, {%1, %2}], [%3];" ::"l"(
                            (uint64_t)&mC),
                        "r"(x), "r"(y), "r"(epi_smem + buf * EPI_BYTES)
                        : "memory");
                    asm volatile("cp.async.bulk.commit_group;" ::: "memory");
                }
            }
            fence_before();
            mbar_arrive(bar(TEMPTY + acc));
        }
        if (issuer) asm volatile("cp.async.bulk.wait_group 0;" ::: "memory");
    }
    __syncthreads();
    if (*abort_flag && threadIdx.x == 0) atomicExch(args.status, 8);
    if (warp == 1) {
        fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem_base), "r"(TMEM_COLS));
    }
}

// ---- operand packing ----------------------------------------------------------------------
__device__ __forceinline__ float tf32_rna(float x) {
    uint32_t r;
    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
    return __uint_as_float(r);
}
__device__ __forceinline__ void split(float x, float& hi, float& lo) {
    hi = tf32_rna(x);
    lo = tf32_rna(x - hi);
}

// Lemb hi/lo (2m x kp floats, row-major): a 32 x 32 complex tile through shared memory.
__global__ void pack_l_kernel(const float2* __restrict__ A, size_t lda, int r0, int k0, int m, int w, int kp,
                              float* __restrict__ hi, float* __restrict__ lo) {
    __shared__ float2 tile[32][33];
    int mu0 = blockIdx.x * 32, k00 = blockIdx.y * 32;
    int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;  // 32 x 8
    for (int r = ty; r < 32; r += 8) {
        int kk = k00 + r, mu = mu0 + tx;
        tile[r][tx] = (kk < w && mu < m) ? A[(size_t)(k0 + kk) * lda + r0 + mu] : make_float2(0.f, 0.f);
    }
    __syncthreads();
    for (int r = ty; r < 32; r += 8) {
        int mu = mu0 + r, kk = k00 + tx;
        if (mu >= m || 2 * kk >= kp) continue;
        float2 l = tile[tx][r];
        float rh, rl, ih, il;
        split(l.x, rh, rl);
        split(l.y, ih, il);
        size_t o0 = (size_t)(2 * mu) * kp + 2 * kk, o1 = o0 + kp;
        *(float2*)(hi + o0) = make_float2(rh, -ih);
        *(float2*)(hi + o1) = make_float2(ih, rh);
        *(float2*)(lo + o0) = make_float2(rl, -il);
        *(float2*)(lo + o1) = make_float2(il, rl);
    }
}

// U hi/lo (n' x kp floats, row-major): row nu = interleaved column nu of U12. lo may be null
// (the two-pass split reads only hi, U12 rounded to TF32).
__global__ void pack_u_kernel(const float2* __restrict__ A, size_t lda, int r0, int k0, int ncols, int w, int kp,
                              float* __restrict__ hi, float* __restrict__ lo) {
    size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    int half = kp / 2;
    if (t >= (size_t)ncols * half) return;
    int nu = (int)(t / half), kk = (int)(t % half);
    float2 u = kk < w ? A[(size_t)(r0 + nu) * lda + k0 + kk] : make_float2(0.f, 0.f);
    float rh, rl, ih, il;
    split(u.x, rh, rl);
    split(u.y, ih, il);
    size_t o = (size_t)nu * kp + 2 * kk;
    *(float2*)(hi + o) = make_float2(rh, ih);
    if (lo) *(float2*)(lo + o) = make_float2(rl, il);
}

// x <- -x over hi and lo halves (2 count floats starting at p, contiguous)
__global__ void negate_kernel(float* __restrict__ p, size_t count) {
    size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t < count) p[t] = -p[t];
}

// ---- FP16 pieces -----------------------------------------------------------------------
// Every row of the A operand (complex row mu of L21, both its real rows) and every row of the
// B operand (column nu of U12) gets its own power-of-two scale f16_scale(max over its K
// entries), so each row's pieces keep 22 bits relative to that row's largest entry.

__device__ __forceinline__ void split16(float x, float s, __half& hi, __half& lo) {
    float xs = x * s;
    hi = __float2half_rn(xs);
    lo = __float2half_rn(xs - __half2float(hi));
}

// Lemb pieces (2m x kp halves, row-major) of 32 complex rows per CTA (K <= 256 real, i.e.
// w <= 128); sign -1 negates. sA[mu] receives the row's scale.
__global__ void __launch_bounds__(256) pack_l16_kernel(const float2* __restrict__ A, size_t lda, int r0, int k0, int m,
                                                       int w, int kp, float sign, __half* __restrict__ hi,
                                                       __half* __restrict__ lo, float* __restrict__ sA) {
    __shared__ float2 tile[128][33];  // [kk][mu]
    __shared__ float scale[32];
    const int mu0 = blockIdx.x * 32, half = kp / 2;
    const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;  // 32 x 8
    for (int kk = ty; kk < half; kk += 8) {
        int mu = mu0 + tx;
        tile[kk][tx] = (kk < w && mu < m) ? A[(size_t)(k0 + kk) * lda + r0 + mu] : make_float2(0.f, 0.f);
    }
    __syncthreads();
    for (int r = ty; r < 32; r += 8) {  // warp ty: rows r; lanes over K
        float mx = 0.0f;
        for (int kk = tx; kk < half; kk += 32) mx = fmaxf(mx, fmaxf(fabsf(tile[kk][r].x), fabsf(tile[kk][r].y)));
        for (int o = 16; o > 0; o >>= 1) mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, o));
        if (tx == 0) {
            float sc = f16_scale(mx);
            scale[r] = sign * sc;
            if (mu0 + r < m) sA[mu0 + r] = sc;
        }
    }
    __syncthreads();
    for (int r = ty; r < 32; r += 8) {
        const int mu = mu0 + r;
        if (mu >= m) continue;
        const float sc = scale[r];
        for (int kk = tx; kk < half; kk += 32) {
            float2 l = tile[kk][r];
            __half rh, rl, ih, il;
            split16(l.x, sc, rh, rl);
            split16(l.y, sc, ih, il);
            size_t o0 = (size_t)(2 * mu) * kp + 2 * kk, o1 = o0 + kp;
            *(__half2*)(hi + o0) = __halves2half2(rh, __hneg(ih));
            *(__half2*)(hi + o1) = __halves2half2(ih, rh);
            *(__half2*)(lo + o0) = __halves2half2(rl, __hneg(il));
            *(__half2*)(lo + o1) = __halves2half2(il, rl);
        }
    }
}

// U pieces (n' x kp halves, row-major): row nu = interleaved column nu of U12; one warp per
// row, sB[nu] its scale.
__global__ void __launch_bounds__(256) pack_u16_kernel(const float2* __restrict__ A, size_t lda, int r0, int k0,
                                                       int ncols, int w, int kp, __half* __restrict__ hi,
                                                       __half* __restrict__ lo, float* __restrict__ sB) {
    const int nu = (int)(((size_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5), lane = threadIdx.x & 31;
    if (nu >= ncols) return;
    const int half = kp / 2;
    float2 u[4];  // kp / 2 <= 128 values per row
    float mx = 0.0f;
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        int kk = lane + 32 * q;
        u[q] = (kk < w && kk < half) ? A[(size_t)(r0 + nu) * lda + k0 + kk] : make_float2(0.f, 0.f);
        mx = fmaxf(mx, fmaxf(fabsf(u[q].x), fabsf(u[q].y)));
    }
    for (int o = 16; o > 0; o >>= 1) mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    const float sc = f16_scale(mx);
    if (lane == 0) sB[nu] = sc;
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        int kk = lane + 32 * q;
        if (kk >= half) continue;
        __half rh, rl, ih, il;
        split16(u[q].x, sc, rh, rl);
        split16(u[q].y, sc, ih, il);
        size_t o = (size_t)nu * kp + 2 * kk;
        *(__half2*)(hi + o) = __halves2half2(rh, ih);
        *(__half2*)(lo + o) = __halves2half2(rl, il);
    }
}

// ---- host -------------------------------------------------------------------------------
typedef CUresult (*EncodeTiled)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

static EncodeTiled encoder() {
    static const EncodeTiled fn = [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            return (EncodeTiled)p;
        return (EncodeTiled) nullptr;
    }();
    return fn;
}

// K-major operand of `rows` rows of kp elements (4-byte TF32 pieces or 2-byte FP16 pieces);
// boxes are one 64-byte swizzle row deep (16 or 32 elements).
static bool make_map(CUtensorMap* map, void* base, int rows, int kp, int box_rows, bool f16) {
    EncodeTiled enc = encoder();
    if (!enc) return false;
    const int eb = f16 ? 2 : 4;
    cuuint64_t dims[2] = {(cuuint64_t)kp, (cuuint64_t)rows};
    cuuint64_t strides[1] = {(cuuint64_t)kp * eb};
    cuuint32_t box[2] = {(cuuint32_t)(64 / eb), (cuuint32_t)box_rows};
    cuuint32_t estr[2] = {1, 1};
    return enc(map, f16 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT16 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, base, dims, strides, box,
               estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_64B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
               CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

__global__ void tri_inverse_l_kernel(const float2* __restrict__ A, size_t lda, int k0, int w, float2* __restrict__ N);
constexpr size_t TI_SMEM = (size_t)(128 * 129 + 64 * 64) * sizeof(float2);

// TF32 pieces by default; FP16 pieces (twice the tensor rate) with TCU_SPLIT=f16. On the
// cluster operators measured here the entries of one row of L21 or one column of U12 span
// more than 2^20 even after equilibration, and FP16 pieces (8 exponent bits fewer) then leave
// the FP64 refinement stalled, so every solve fell back to TF32 pieces.
// Two passes hi*hi + lo*hi (the B operand, U12, rounded to TF32) unless TCU_SPLIT asks for
// three TF32 passes (tf32x3) or FP16 pieces (f16): a third fewer tensor-core passes and no B lo
// loads, for an update accurate to about 2^-11 relative to max|A| max|B| per term. The FP64
// refinement then takes one sweep more (512 spheres lmax 4: 3 instead of 2, factor 279 instead
// of 320 ms), and a stall falls back to the three-pass factor.
bool split_two_pass_default() {
    static const bool on = [] {
        const char* e = getenv("TCU_SPLIT");
        return !(e && (std::strcmp(e, "tf32x3") == 0 || std::strcmp(e, "f16") == 0));
    }();
    return on;
}

bool split_f16_default() {
    static const bool on = [] {
        const char* e = getenv("TCU_SPLIT");
        return e && std::strcmp(e, "f16") == 0;
    }();
    return on;
}

bool tf32_enabled() {
    static const int on = [] {
        const char* e = getenv("TCU_DISABLE_TCGEN05");
        return (e && e[0] == '1') || !encoder() ? 0 : 1;
    }();
    if (on == 1) {
        static PerDeviceOnce attr;
        once_per_device(attr, [] {
            cudaFuncSetAttribute(tf32_update_kernel<false, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)TF32_SMEM);
            cudaFuncSetAttribute(tf32_update_kernel<false, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)TF32_SMEM);
            cudaFuncSetAttribute(tf32_update_kernel<true, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)TF32_SMEM);
            cudaFuncSetAttribute(tri_inverse_l_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)TI_SMEM);
        });
    }
    return on == 1;
}

// N = L11^-1 - I for the unit lower w x w (w <= 128) diagonal block of the panel, in FP32
// in shared memory, by recursive doubling: the eight 16 x 16 diagonal blocks are inverted
// by one warp each (columns right to left), then pairs of inverted blocks [A 0; B C] are
// joined level by level (s = 16, 32, 64) with the lower-left block -C^-1 B A^-1 formed as
// two small dense products. M holds the strictly lower part; unit diagonals are implicit.
// Stored column-major w x w. U12 = L11^-1 A12 = A12 + N A12 then runs on the tensor cores.
__device__ __forceinline__ float2 cmulf(float2 a, float2 b) {
    return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__global__ void __launch_bounds__(1024) tri_inverse_l_kernel(const float2* __restrict__ A, size_t lda, int k0, int w,
                                                            float2* __restrict__ N) {
    extern __shared__ float2 ti_smem[];
    const int LD = 129;
    float2* M = ti_smem;             // M[i * LD + k], 128 x 128
    float2* T = ti_smem + 128 * LD;  // 64 x 64 scratch
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    for (int idx = tid; idx < 128 * 128; idx += blockDim.x) {
        int i = idx % 128, k = idx / 128;
        M[i * LD + k] = (i > k && i < w && k < w) ? A[(size_t)(k0 + k) * lda + k0 + i] : make_float2(0.f, 0.f);
    }
    __syncthreads();
    // 16 x 16 diagonal blocks: X[i][j] = -sum_{k=j+1..i} X[i][k] L[k][j], X[i][i] = 1
    if (warp < 8) {  // one warp per 16 x 16 block; the other warps join at the next barrier
        __shared__ float2 colbuf[8][16];
        const int o = warp * 16;
        for (int j = 14; j >= 0; --j) {
            if (lane < 16) colbuf[warp][lane] = M[(o + lane) * LD + o + j];
            __syncwarp();
            if (lane < 16 && lane > j) {
                int i = lane;
                float2 sum = colbuf[warp][i];  // k = i term
                for (int k = j + 1; k < i; ++k) {
                    float2 l = colbuf[warp][k], x = M[(o + i) * LD + o + k];
                    sum.x += x.x * l.x - x.y * l.y;
                    sum.y += x.x * l.y + x.y * l.x;
                }
                M[(o + i) * LD + o + j] = make_float2(-sum.x, -sum.y);
            }
            __syncwarp();
        }
    }
    __syncthreads();
    // join pairs: [A 0; B C]^-1 lower-left = -Cinv (B Ainv)
    for (int s = 16; s < 128; s *= 2) {
        const int pairs = 128 / (2 * s);
        // T = B Ainv for every pair (pair p stores at T + p * s * s)
        for (int idx = tid; idx < pairs * s * s; idx += blockDim.x) {
            int p = idx / (s * s), e = idx % (s * s), i = e / s, k = e % s;
            int a0 = p * 2 * s, c0 = a0 + s;
            float2 sum = M[(c0 + i) * LD + a0 + k];  // m = k, Ainv diagonal 1
            for (int m = k + 1; m < s; ++m) {
                float2 b = M[(c0 + i) * LD + a0 + m], x = M[(a0 + m) * LD + a0 + k];
                sum.x += b.x * x.x - b.y * x.y;
                sum.y += b.x * x.y + b.y * x.x;
            }
            T[p * s * s + i * s + k] = sum;
        }
        __syncthreads();
        // lower-left = -(Cinv T)
        for (int idx = tid; idx < pairs * s * s; idx += blockDim.x) {
            int p = idx / (s * s), e = idx % (s * s), i = e / s, k = e % s;
            int a0 = p * 2 * s, c0 = a0 + s;
            float2 sum = T[p * s * s + i * s + k];  // m = i, Cinv diagonal 1
            for (int m = 0; m < i; ++m) {
                float2 c = M[(c0 + i) * LD + c0 + m], t = T[p * s * s + m * s + k];
                sum.x += c.x * t.x - c.y * t.y;
                sum.y += c.x * t.y + c.y * t.x;
            }
            M[(c0 + i) * LD + a0 + k] = make_float2(-sum.x, -sum.y);
        }
        __syncthreads();
    }
    for (int idx = tid; idx < w * w; idx += blockDim.x) {
        int ii = idx % w, k = idx / w;
        N[(size_t)k * w + ii] = M[ii * LD + k];
    }
}
size_t tf32_pack_bytes(int n) {
    size_t kp = 512;  // two 128-column panels per trailing update
    return ((size_t)2 * n * kp + (size_t)n * kp) * 2 * 4 + (size_t)128 * 128 * 8 + 8192;
}

static int num_sms() {
    static const int sms = [] {
        int dev = 0, v = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev);
        return v;
    }();
    return sms;
}

// The packed operands live in the buffer the factor allocated from its context's pool
// (tf32_pack_bytes(n), enough for every step of an n x n factorization); a step that would
// need more records status 6 (out of memory) instead of reallocating outside the pool.
static bool ensure_pack(LuWork& wk, size_t need, cudaStream_t st) {
    if (wk.pack && wk.pack_bytes >= need) return true;
    cudaMemsetAsync(wk.status, 6, 1, st);
    return false;
}

// C[row0 .. row0+m2) x [col0 .. col0+ncols) -= Apack (m2 x kp) * Bpack (ncols x kp)^T;
// sA != null selects FP16 pieces (row scales sA of the A operand, sB of the B operand).
static void run_gemm(float2* A, int n, int row0, int col0, int m2, int ncols, int kp, void* ahi, void* alo, void* bhi,
                     void* blo, const float* sA, const float* sB, LuWork& wk, cudaStream_t st, long long* launches,
                     bool two = false) {
    const bool f16 = sA != nullptr;
    CUtensorMap mAhi, mAlo, mBhi, mBlo;
    bool ok = make_map(&mAhi, ahi, m2, kp, TB_M, f16) && make_map(&mAlo, alo, m2, kp, TB_M, f16) &&
              make_map(&mBhi, bhi, ncols, kp, TB_N, f16) && make_map(&mBlo, blo, ncols, kp, TB_N, f16);
    // A viewed as a 2n x n float matrix (column-major): box of 128 real rows x 64 columns
    CUtensorMap mC;
    {
        EncodeTiled enc = encoder();
        cuuint64_t dims[2] = {(cuuint64_t)2 * n, (cuuint64_t)n};
        cuuint64_t strides[1] = {(cuuint64_t)2 * n * 4};
        cuuint32_t box[2] = {(cuuint32_t)TB_M, (cuuint32_t)EPI_COLS};
        cuuint32_t estr[2] = {1, 1};
        ok = ok && enc && enc(&mC, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, (void*)A, dims, strides, box, estr,
                              CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                              CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
    }
    if (!ok) {
        cudaMemsetAsync(wk.status, 7, 1, st);
        return;
    }
    Tf32Args a;
    a.C = (float*)A;
    a.ldc = (size_t)2 * n;
    a.row0 = row0;
    a.col0 = col0;
    a.m2 = m2;
    a.ncols = ncols;
    a.kchunks = kp / (f16 ? 32 : TB_K);
    a.tiles_m = (m2 + TB_M - 1) / TB_M;
    a.tiles_n = (ncols + TB_N - 1) / TB_N;
    a.tiles = a.tiles_m * a.tiles_n;
    a.status = wk.status;
    a.sA = sA;
    a.sB = sB;
    int grid = std::min(num_sms(), a.tiles);
    if (f16)
        tf32_update_kernel<true, false><<<grid, 192, TF32_SMEM, st>>>(mAhi, mAlo, mBhi, mBlo, mC, a);
    else if (two)
        tf32_update_kernel<false, true><<<grid, 192, TF32_SMEM, st>>>(mAhi, mAlo, mBhi, mBlo, mC, a);
    else
        tf32_update_kernel<false, false><<<grid, 192, TF32_SMEM, st>>>(mAhi, mAlo, mBhi, mBlo, mC, a);
    *launches += 1;
}

// U12 = L11^-1 A12 on the tensor cores: invert L11, then A12 -= (-(L11^-1 - I)) A12 with the
// operands packed (A12 is read from its packed copy, so the in-place update is race free).
// Operand buffer of one TRSM step (sized on the host; a reallocation synchronises the device)
// and the place of N = L11^-1 - I in it; null when it could not be sized.
static float2* trsm_buffers(int n, int k0, int w, LuWork& wk, cudaStream_t st, int* kp_out) {
    int r0 = k0 + w, ncols = n - r0;
    int kp = ((2 * w + 31) / 32) * 32;  // whole 64-byte K rows of FP16 pieces (and of TF32)
    size_t need = ((size_t)2 * w * kp + (size_t)ncols * kp) * 2 * 4 + (size_t)w * w * 8 + 8192;
    if (!ensure_pack(wk, need, st)) return nullptr;
    *kp_out = kp;
    float* blo = (float*)wk.pack + (size_t)4 * w * kp + (size_t)ncols * kp;
    return (float2*)(((uintptr_t)(blo + (size_t)ncols * kp) + 255) & ~(uintptr_t)255);
}

bool launch_tf32_trsm_inverse(float2* A, int n, int k0, int w, LuWork& wk, cudaStream_t st, cudaStream_t side,
                              long long* launches) {
    int kp;
    float2* Nm = trsm_buffers(n, k0, w, wk, st, &kp);
    if (!Nm) return false;
    tri_inverse_l_kernel<<<1, 1024, TI_SMEM, side>>>(A, (size_t)n, k0, w, Nm);
    ++*launches;
    // a refused launch leaves the inverse to the main stream (launch_tf32_trsm, inverse_done false)
    return cudaGetLastError() == cudaSuccess;
}

// The TRSM's right-hand side A12 as TF32 pieces, packed before the main stream waits for the
// inverse of L11 (which it does not need); launch_tf32_trsm(..., rhs_packed = true) then skips
// it. FP16 pieces keep their packing in launch_tf32_trsm (false here).
bool launch_tf32_trsm_rhs(float2* A, int n, int k0, int w, LuWork& wk, cudaStream_t st, long long* launches) {
    if (wk.f16_pieces) return false;
    int r0 = k0 + w, ncols = n - r0, kp;
    if (ncols <= 0 || !trsm_buffers(n, k0, w, wk, st, &kp)) return false;
    float* bhi = (float*)wk.pack + (size_t)4 * w * kp;
    float* blo = bhi + (size_t)ncols * kp;
    StageScope sc(ST_TRSM, st);
    size_t tot = (size_t)ncols * (kp / 2);
    pack_u_kernel<<<(unsigned)((tot + 255) / 256), 256, 0, st>>>(A, (size_t)n, r0, k0, ncols, w, kp, bhi, blo);
    ++*launches;
    return true;
}

void launch_tf32_trsm(float2* A, int n, int k0, int w, LuWork& wk, cudaStream_t st, long long* launches,
                      bool inverse_done, bool rhs_packed) {
    int r0 = k0 + w, ncols = n - r0;
    int kp;
    float2* Nm = trsm_buffers(n, k0, w, wk, st, &kp);
    if (!Nm) return;
    float* ahi = (float*)wk.pack;
    float* alo = ahi + (size_t)2 * w * kp;
    float* bhi = alo + (size_t)2 * w * kp;
    float* blo = bhi + (size_t)ncols * kp;
    {
        StageScope sc(ST_TRSM, st);
        if (!inverse_done) {
            tri_inverse_l_kernel<<<1, 1024, TI_SMEM, st>>>(A, (size_t)n, k0, w, Nm);
            if (cudaGetLastError() != cudaSuccess) {  // U12 would use a stale inverse: stop the factorization
                cudaMemsetAsync(wk.status, 7, 1, st);
                return;
            }
        }
        dim3 g1((w + 31) / 32, (kp / 2 + 31) / 32);
        size_t tot = (size_t)ncols * (kp / 2);
        if (wk.f16_pieces) {
            // A operand: -N embedded, so that the update C -= (-N) A12 adds N A12
            __half *h_ahi = (__half*)ahi, *h_alo = h_ahi + (size_t)2 * w * kp;
            __half *h_bhi = h_alo + (size_t)2 * w * kp, *h_blo = h_bhi + (size_t)ncols * kp;
            float* sA = (float*)(((uintptr_t)(h_blo + (size_t)ncols * kp) + 255) & ~(uintptr_t)255);
            float* sB = (float*)(((uintptr_t)(sA + w) + 255) & ~(uintptr_t)255);
            pack_l16_kernel<<<(w + 31) / 32, 256, 0, st>>>(Nm, (size_t)w, 0, 0, w, w, kp, -1.0f, h_ahi, h_alo, sA);
            pack_u16_kernel<<<(unsigned)(((size_t)ncols * 32 + 255) / 256), 256, 0, st>>>(A, (size_t)n, r0, k0, ncols, w,
                                                                                         kp, h_bhi, h_blo, sB);
            run_gemm(A, n, 2 * k0, r0, 2 * w, ncols, kp, h_ahi, h_alo, h_bhi, h_blo, sA, sB, wk, st, launches);
            *launches += 3;
        } else {
            pack_l_kernel<<<g1, 256, 0, st>>>(Nm, (size_t)w, 0, 0, w, w, kp, ahi, alo);
            if (!rhs_packed) {
                pack_u_kernel<<<(unsigned)((tot + 255) / 256), 256, 0, st>>>(A, (size_t)n, r0, k0, ncols, w, kp, bhi,
                                                                             blo);
                ++*launches;
            }
            negate_kernel<<<(unsigned)(((size_t)4 * w * kp + 255) / 256), 256, 0, st>>>(ahi, (size_t)4 * w * kp);
            run_gemm(A, n, 2 * k0, r0, 2 * w, ncols, kp, ahi, alo, bhi, blo, nullptr, nullptr, wk, st, launches);
            *launches += 3;
        }
    }
}

// A[r0 .. r0+m) x [c0 .. c0+ncols) -= A[r0.., k0 .. k0+w) A[k0 .. k0+w, c0..): the trailing
// update of panel columns k0 .. k0+w restricted to a block of rows and columns.
void launch_tf32_update_region(float2* A, int n, int k0, int w, int r0, int m, int c0, int ncols, LuWork& wk,
                               cudaStream_t st, long long* launches) {
    if (m <= 0 || ncols <= 0) return;
    int kp = ((2 * w + 31) / 32) * 32;  // whole 64-byte K rows of FP16 pieces (and of TF32)
    size_t need = ((size_t)2 * m * kp + (size_t)ncols * kp) * 2 * 4 + 4096;
    if (!ensure_pack(wk, need, st)) return;
    float* ahi = (float*)wk.pack;
    float* alo = ahi + (size_t)2 * m * kp;
    float* bhi = alo + (size_t)2 * m * kp;
    float* blo = bhi + (size_t)ncols * kp;
    const bool f16 = wk.f16_pieces;
    __half *h_ahi = (__half*)ahi, *h_alo = h_ahi + (size_t)2 * m * kp;
    __half *h_bhi = h_alo + (size_t)2 * m * kp, *h_blo = h_bhi + (size_t)ncols * kp;
    float* sA = (float*)(((uintptr_t)(h_blo + (size_t)ncols * kp) + 255) & ~(uintptr_t)255);
    float* sB = (float*)(((uintptr_t)(sA + m) + 255) & ~(uintptr_t)255);
    {
        StageScope sc(ST_PACK, st);
        if (f16) {
            pack_l16_kernel<<<(m + 31) / 32, 256, 0, st>>>(A, (size_t)n, r0, k0, m, w, kp, 1.0f, h_ahi, h_alo, sA);
            pack_u16_kernel<<<(unsigned)(((size_t)ncols * 32 + 255) / 256), 256, 0, st>>>(A, (size_t)n, c0, k0, ncols, w,
                                                                                         kp, h_bhi, h_blo, sB);
        } else {
            dim3 g1((m + 31) / 32, (kp / 2 + 31) / 32);
            size_t tot = (size_t)ncols * (kp / 2);
            pack_l_kernel<<<g1, 256, 0, st>>>(A, (size_t)n, r0, k0, m, w, kp, ahi, alo);
            pack_u_kernel<<<(unsigned)((tot + 255) / 256), 256, 0, st>>>(A, (size_t)n, c0, k0, ncols, w, kp, bhi,
                                                                         wk.two_pass ? nullptr : blo);
        }
        *launches += 2;
    }
    StageScope sc(ST_GEMM, st);
    if (f16)
        run_gemm(A, n, 2 * r0, c0, 2 * m, ncols, kp, h_ahi, h_alo, h_bhi, h_blo, sA, sB, wk, st, launches);
    else
        run_gemm(A, n, 2 * r0, c0, 2 * m, ncols, kp, ahi, alo, bhi, blo, nullptr, nullptr, wk, st, launches,
                 wk.two_pass);
}

void launch_tf32_update(float2* A, int n, int k0, int w, LuWork& wk, cudaStream_t st, long long* launches) {
    const int r0 = k0 + w;
    launch_tf32_update_region(A, n, k0, w, r0, n - r0, r0, n - r0, wk, st, launches);
}

}  // namespace tcu
