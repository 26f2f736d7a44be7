// Host-side launchers of the device kernels (one header for the C ABI layer).
#pragma once
#include <cuda_runtime.h>
#include <stddef.h>

#include "../../include/treams_cuda.h"
#include "plan.h"

#include <atomic>
#include <mutex>
#include <vector>

namespace tcu {

typedef double2 cplx;

// Kernel attributes (large dynamic shared memory) are per device: each site keeps one bit per
// device in `mask`, and this returns true the first time it runs with that device current.
struct PerDeviceOnce {
    std::mutex mu;
    unsigned long long done = 0;  // bit d: done on device d
};
// Runs f once per process and current device; callers on other threads wait until it is done
// (the batched solve launches from several host threads).
template <class F>
inline void once_per_device(PerDeviceOnce& o, F&& f) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) {
        f();
        return;
    }
    const unsigned long long bit = 1ull << dev;
    std::lock_guard<std::mutex> g(o.mu);
    if (o.done & bit) return;
    f();
    o.done |= bit;
}

// Per-stage CUDA-event timing (tcu_context_set_profiling). The API layer installs the
// context's profiler as the calling thread's current one for the duration of a call; the
// launch sites bracket their kernels with a StageScope.
enum Stage { ST_ASSEMBLE = 0, ST_PANEL, ST_SWAP, ST_TRSM, ST_GEMM, ST_PACK, ST_SOLVE, ST_APPLY, ST_MIE, ST_LATTICE,
             ST_SMALL_LU, ST_COARSE, ST_NEAR, ST_COUNT };
struct Profiler {
    bool on = false;
    struct Rec {
        int stage;
        cudaEvent_t a, b;
    };
    std::vector<Rec> recs;
    std::vector<cudaEvent_t> pool;
    double total_ms[ST_COUNT] = {};
    long long count[ST_COUNT] = {};
    cudaEvent_t take() {
        if (!pool.empty()) {
            cudaEvent_t e = pool.back();
            pool.pop_back();
            return e;
        }
        cudaEvent_t e;
        cudaEventCreate(&e);
        return e;
    }
    void collect() {
        for (auto& r : recs) {
            cudaEventSynchronize(r.b);
            float ms = 0.f;
            cudaEventElapsedTime(&ms, r.a, r.b);
            total_ms[r.stage] += ms;
            count[r.stage] += 1;
            pool.push_back(r.a);
            pool.push_back(r.b);
        }
        recs.clear();
    }
    ~Profiler() {
        collect();
        for (auto e : pool) cudaEventDestroy(e);
    }
};
extern thread_local Profiler* g_prof;

// Device memory of objects that live within one API call (preconditioners, their graphs and
// coarse solvers): the context's caching pool while the call has installed it (PoolScope),
// else cudaMalloc / cudaFree. Each allocation remembers where it came from.
struct DeviceAllocator {
    virtual cudaError_t alloc(void** p, size_t bytes) = 0;
    virtual void release(void* p) = 0;

   protected:
    ~DeviceAllocator() = default;
};
extern thread_local DeviceAllocator* g_call_pool;
struct PoolScope {
    DeviceAllocator* prev;
    explicit PoolScope(DeviceAllocator* a) : prev(g_call_pool) { g_call_pool = a; }
    ~PoolScope() { g_call_pool = prev; }
};
inline cudaError_t call_malloc(void** p, size_t bytes, DeviceAllocator** owner) {
    *owner = g_call_pool;
    return *owner ? (*owner)->alloc(p, bytes) : cudaMalloc(p, bytes);
}
inline void call_free(void* p, DeviceAllocator* owner) {
    if (!p) return;
    if (owner)
        owner->release(p);
    else
        cudaFree(p);
}
struct StageScope {
    Profiler* p;
    int stage;
    cudaStream_t st;
    cudaEvent_t a = nullptr;
    StageScope(int stage_, cudaStream_t st_) : p(g_prof), stage(stage_), st(st_) {
        if (p && p->on) {
            a = p->take();
            cudaEventRecord(a, st);
        }
    }
    ~StageScope() {
        if (a) {
            cudaEvent_t b = p->take();
            cudaEventRecord(b, st);
            p->recs.push_back({stage, a, b});
        }
    }
};

// pairs.cu
void launch_assemble(const DevPlan& P, int N, double k, const double* pos, const cplx* T, void* out, size_t ld,
                     bool fp32, cudaStream_t st);
void launch_apply(const DevPlan& P, int N, double k, const double* pos, const cplx* T, const cplx* x, size_t ldx,
                  int ncol, const cplx* zadd, double alpha, double beta, bool singular, cplx* y, cudaStream_t st);
size_t apply_smem_bytes(const DevPlan& P, int ncol);
// Product form of the same operator (lmax 2..5; TCU_APPLY=terms selects the term-sum kernels)
bool apply_gemm_supported(const DevPlan& P);
void launch_apply_gemm(const DevPlan& P, int N, double k, const double* pos, const cplx* T, const cplx* x, size_t ldx,
                       int ncol, const cplx* zadd, double alpha, double beta, bool singular, cplx* y, cudaStream_t st);
void apply_gemm_init_attributes();
// Dipole blocks of the operator in product form, one vector: z holds the 6 dipole modes of every
// sphere; y = zadd + alpha (z on the dipole modes) + beta T (C P z), on all modes (y: n) or, with
// dipole_rows, on the dipole modes only (y: 6N). P z is z on the dipole modes, zero elsewhere.
void launch_apply_dipole(const DevPlan& P, int N, double k, const double* pos, const cplx* T, const cplx* z,
                         bool dipole_rows, const cplx* zadd, double alpha, double beta, cplx* y, cudaStream_t st);
// Stored-table form of the singular operator and of its two dipole blocks (for repeated
// applications): the harmonic tables of all ordered pairs built once into Z
// (stored_tables_bytes), then every application is an FP64 tensor-core product over Z plus the
// term lists. kind: STORED_FULL (lmax 2..5) is launch_apply's operator; STORED_DIPOLE_SOURCES and
// STORED_DIPOLE_BLOCK are launch_apply_dipole with dipole_rows false and true (input ldin 6).
// Xf: scratch of stored_inputs_bytes for the packed inputs. Sizes are 0 where a kind does not
// apply.
enum StoredKind { STORED_FULL = 0, STORED_DIPOLE_SOURCES = 1, STORED_DIPOLE_BLOCK = 2 };
bool stored_tables_enabled();  // false when TCU_APPLY is "fly" or "terms" (read at every call)
size_t stored_tables_bytes(const DevPlan& P, int N, int kind);
size_t stored_inputs_bytes(const DevPlan& P, int N, int kind, int ncol);
void build_stored_tables(const DevPlan& P, int N, double k, const double* pos, int kind, cplx* Z, cudaStream_t st);
// status (may be null) receives 8 when a bounded wait of the product gave up (y not written).
void launch_apply_stored(const DevPlan& P, int N, int kind, const cplx* Z, const cplx* T, const cplx* x, size_t ldx,
                         int ncol, const cplx* zadd, double alpha, double beta, cplx* y, cplx* Xf, int* status,
                         cudaStream_t st);
void launch_block(const DevPlan& P, double k, const double* d, bool singular, bool helicity, cplx* out,
                  cudaStream_t st);
void launch_mie(int L, double k0, int N, const double* radii, const cplx* eps, cplx* T, int* status, cudaStream_t st);
void launch_plane_wave(int L, int N, const double* pos, int ncol, const cplx* kvecs, const int* pols,
                       const double* lfac, cplx* out, cudaStream_t st);
void launch_apply_t(int L, int N, const cplx* T, const cplx* x, int ncol, cplx* y, cudaStream_t st);
// regular translation blocks between the N spheres (nlm_loc lm per sphere) and the origin
// (nlm_glob lm), cut from blocks of the plan P (P.nlm >= both): Ein n x Mg, Eout Mg x n
// (cleared by the caller); and a small complex FP64 GEMM C = A B (column-major)
void launch_expand_blocks(const DevPlan& P, int N, double k, const double* pos, const double* origin, int nlm_loc,
                          int nlm_glob, cplx* Ein, cplx* Eout, cudaStream_t st);
void launch_zgemm_small(int m, int n, int k, const cplx* A, size_t lda, const cplx* B, size_t ldb, cplx* C,
                        size_t ldc, cudaStream_t st);
void pairs_init_attributes();
// translate.cu — per-entry translation coefficients: labels 6 ints per element (lambda, mu,
// pol, l, m, qol), args 3 complex per element (kr, theta, phi)
void launch_translate(const DevPlan& P, size_t count, const int* labels, const cplx* args, bool helicity,
                      bool singular, cplx* out, cudaStream_t st);

// adjoint.cu — y = (I - T C)^H x for ncol columns of leading dimension ldx (t1, t2: ldx x ncol
// scratch; with stored pair tables Z (STORED_FULL) the coupling product runs over them, Xf:
// stored_inputs_bytes for ncol columns, status as for launch_apply_stored), y = T^H x, and
// x <- A^-H x with the LU factors (tmp: adjoint_solve_tmp(n, ncol))
void launch_apply_adjoint(const DevPlan& P, int N, double k0, const double* pos, const cplx* T, const cplx* x,
                          size_t ldx, int ncol, cplx* y, cplx* t1, cplx* t2, cudaStream_t st, long long* launches,
                          const cplx* Z = nullptr, cplx* Xf = nullptr, int* status = nullptr);
void launch_apply_th(int L, int N, const cplx* T, const cplx* x, size_t ldx, int ncol, cplx* y, cudaStream_t st);
size_t adjoint_solve_tmp(int n, int ncol);
void lu_solve_adjoint_fp64(const double2* A, int n, const int* perm, const double2* inv, double2* x, double2* tmp,
                           int ncol, cudaStream_t st, long long* launches);
void lu_solve_adjoint_fp32(const float2* A, int n, const int* perm, const double2* inv, double2* x, double2* tmp,
                           int ncol, cudaStream_t st, long long* launches);

// equil.cu — power-of-two row/column equilibration of an n x n column-major matrix (FP64 or
// FP32 storage) when its largest entry exceeds `threshold`; r, c: n scales each.
size_t equilibrate_scratch_doubles(int n);
tcu_status equilibrate(void* A, bool fp32, int n, double threshold, double* r, double* c, double* partial,
                       bool* applied, cudaStream_t st, long long* launches);
void scale_rows(cplx* v, const double* s, size_t n, int ncol, cudaStream_t st);

// lattice.cu — 2D lattice sums (any real shift) and the batched periodic-array solve
constexpr int LS_MAXL = 14;                // largest degree of a lattice sum
constexpr int LS_NMAX = LS_MAXL / 2 + 1;   // reciprocal orders n per (l, m) in the plane
constexpr int LS_FMAX = LS_MAXL + 1;       // reciprocal orders n per (l, m) off the plane
constexpr int LS_PMAX = LS_MAXL / 2 + 1;   // powers of beta^2 in S_lmn off the plane
constexpr int LS_TMAX = 64;                // most terms of the t-series of F_(1/2-n)(v, t)
struct LatticeSumArgs {
    int lsum = 0;                          // degrees l <= lsum, T = (lsum+1)^2 outputs
    double k = 0, eta = 0;
    int NR = 0;                            // real-space lattice points (R != 0)
    const double2* R = nullptr;
    const double2* realtab = nullptr;      // NR x T real-space terms
    int NG = 0;                            // reciprocal lattice vectors
    const double2* G = nullptr;
    const double2* Glo = nullptr;          // their low parts (G = G + Glo to twice FP64 precision)
    const double* coef = nullptr;          // T x LS_NMAX in-plane polynomial coefficients
    const double2* pref = nullptr;         // T reciprocal prefactors
    double2 self0{0, 0};                   // self term of l = 0 (zero for a nonzero shift)
    double sx = 0, sy = 0;                 // in-plane shift r' (reciprocal phase e^{-i q.r'})
    double R0x = 0, R0y = 0;               // lattice vector taken off the shift: e^{-i kpar.R0}
    // shift off the plane (r_z != 0): every order n <= lsum, F'_n from the t-series of
    // F_(1/2-n)(v, t) with t = (k r_z eta)^2 (J + 1 terms), and S_lmn as a polynomial in beta^2
    // with coefficients coefz[(lm * LS_PMAX + p) * LS_FMAX + n] (powers of -k r_z folded in)
    int offplane = 0;
    int J = 0;
    double t = 0;
    const double* coefz = nullptr;
    int nk = 0;
    const double2* kpar = nullptr;
    double2* out = nullptr;                // out[kp * ldo + l*l+l+m]
    size_t ldo = 0;
    int* status = nullptr;                 // 9: a diffraction order on its threshold
};
// lattice_ck.cu — the same sums at a complex wavenumber (Im k >= 0), any shift, real split
struct LatticeSumCkArgs {
    int lsum = 0;
    double2 k{0, 0};
    double eta = 0;
    int NR = 0;
    const double2* R = nullptr;
    const double2* realtab = nullptr;      // NR x T real-space terms
    int NG = 0;
    const double2* G = nullptr;
    const double2* Glo = nullptr;          // low parts of the reciprocal vectors
    const double2* coef = nullptr;         // T x LS_PMAX x LS_FMAX: S_lmn coefficient of beta^(2p), order n
    const double2* pref = nullptr;         // T reciprocal prefactors (1/k^2 included)
    double2 self0{0, 0};
    double sx = 0, sy = 0, R0x = 0, R0y = 0;
    int J = 0;                             // t-series terms (0 in the plane)
    double2 t{0, 0};                       // (k r_z eta)^2
    double2 ksq{0, 0};                     // k^2
    double turn = 0, near = 0;             // sheet split: arg (k eta)^2, tan^2 of the near sector
    int has_near = 0;
    int nk = 0;
    const double2* kpar = nullptr;
    double2* out = nullptr;
    size_t ldo = 0;
    int* status = nullptr;                 // 9: a diffraction order on its threshold
};
void launch_real_table_ck(int lsum, double2 k, double eta, int NR, const double2* R, double sx, double sy, double sz,
                          const double* norm, const double* reflection, double2* tab, cudaStream_t st);
size_t lattice_sum_ck_smem(int lsum, int NR);
void launch_lattice_sum_ck(const LatticeSumCkArgs& a, int grid, cudaStream_t st);
void launch_real_table(int lsum, double k, double eta, int NR, const double2* R, double sx, double sy, double sz,
                       const double* norm, const double* reflection, double2* tab, cudaStream_t st);
size_t lattice_sum_smem(int lsum, int NR, bool offplane);
void launch_lattice_sum(const LatticeSumArgs& a, int grid, cudaStream_t st);
void launch_array_solve(const DevPlan& P, const double2* D, size_t ldd, const double* norm, const double2* Tm, int nk,
                        double2* X, int* status, int grid, cudaStream_t st);

// lu.cu — dense LU of an n x n column-major complex matrix (lda = n) in FP64 (double2)
// or FP32 (float2) storage, row permutation kept as perm (row i of P A is row perm[i]).
struct LuWork {
    int* piv = nullptr;        // n
    int* perm = nullptr;       // n
    unsigned* barrier = nullptr;
    int* status = nullptr;     // device status word
    void* cand = nullptr;      // candidate values/rows, double-buffered
    void* pack = nullptr;      // packed GEMM operands (mixed path)
    size_t pack_bytes = 0;
    bool f16_pieces = false;   // mixed path: FP16 (true) or TF32 (false) pieces of the 3-pass split
    bool two_pass = false;     // mixed path: two-pass TF32 trailing updates (B operand rounded to TF32)
    int panel_rows = 0;        // least rows per panel CTA (0: TCU_PANEL_ROWS or 32)
};
// FP16 pieces when the environment asks for them (TCU_SPLIT=f16), else TF32 pieces
bool split_f16_default();
// Two-pass TF32 trailing updates unless the environment asks for three passes or FP16 pieces
bool split_two_pass_default();
int lu_factor_fp64(double2* A, int n, LuWork& w, cudaStream_t st, long long* launches);
// The panel's grid barrier with one arrival missing (bar: a zeroed counter); it gives up
// after limit_s (clamped to [0, 4] s) and records status 8.
void launch_barrier_selftest(unsigned* bar, int* status, double limit_s, cudaStream_t st);
int lu_factor_fp32(float2* A, int n, LuWork& w, cudaStream_t st, long long* launches, bool tensor_cores);
// solve.cu — inverses of the 64 x 64 diagonal blocks of L and U (FP64, lu_inverse_bytes),
// then x (n x ncol, FP64) <- A^-1 x; tmp holds 2 n min(ncol, 8) complex.
size_t lu_inverse_bytes(int n);
void lu_block_inverses_fp64(const double2* A, int n, double2* inv, cudaStream_t st, long long* launches);
void lu_block_inverses_fp32(const float2* A, int n, double2* inv, cudaStream_t st, long long* launches);
// epoch: the factor's sweep counter (host), status: its device status word (8 when a sweep's
// bounded wait gave up); both null select one launch per block step.
void lu_solve_fp64(const double2* A, int n, const int* perm, const double2* inv, double2* x, double2* tmp, int ncol,
                   cudaStream_t st, long long* launches, unsigned* epoch = nullptr, int* status = nullptr);
void lu_solve_fp32(const float2* A, int n, const int* perm, const double2* inv, double2* x, double2* tmp, int ncol,
                   cudaStream_t st, long long* launches, unsigned* epoch = nullptr, int* status = nullptr);
size_t lu_workspace_bytes(int n, bool fp32);
size_t tf32_pack_bytes(int n);  // packed tensor-core operands of the mixed LU
void lu_init_attributes();

// blas.cu — fixed-order reductions and vector updates on FP64 complex vectors
void vec_norms(const cplx* x, size_t n, int ncol, double* out_dev, double* partial, cudaStream_t st);
void vec_axpy(cplx* y, const cplx* x, size_t n, int ncol, cudaStream_t st);
void vec_sub(cplx* out, const cplx* a, const cplx* b, size_t n, int ncol, cudaStream_t st);
void vec_dots(const cplx* V, size_t ldv, int nv, const cplx* w, size_t n, cplx* out_dev, cplx* partial,
              cudaStream_t st);
void vec_gemv_sub(cplx* w, const cplx* V, size_t ldv, int nv, const cplx* h_dev, size_t n, cudaStream_t st);
void vec_scale_copy(cplx* out, const cplx* x, size_t n, double s, cudaStream_t st);
void vec_lincomb(cplx* x, const cplx* V, size_t ldv, int nv, const cplx* g_dev, size_t n, cudaStream_t st);
void vec_real_dots(const cplx* a, const cplx* b, size_t n, int ncol, double* out_dev, double* partial,
                   cudaStream_t st);

}  // namespace tcu
