// The C ABI (include/treams_cuda.h): contexts, validation mirroring treams-core, device
// buffers, the dense factor + refinement driver and the GMRES driver.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <complex>
#include <cstdio>
#include <cstring>
#include <functional>
#include <map>
#include <set>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "../../include/treams_cuda.h"
#include "kernels.h"
#include "plan.h"
#include "precond.h"

using namespace tcu;

namespace {

thread_local std::string g_last_error;

tcu_status fail(tcu_status st, const std::string& msg) {
    g_last_error = msg;
    return st;
}

// Caching device allocator of a context: blocks freed by factors and per-call buffers are
// kept for reuse (stream-ordered on the context's stream), so repeated factorizations do
// not pay cudaMalloc/cudaFree of multi-GB matrices. Pooled blocks are released on
// allocation failure and when the context is destroyed.
struct DevicePool : tcu::DeviceAllocator {
    std::multimap<size_t, void*> free_;
    std::map<void*, size_t> sizes_;
    cudaError_t alloc(void** p, size_t bytes) override { return take(p, bytes); }
    void release(void* p) override { free(p); }
    cudaError_t take(void** p, size_t bytes) {
        bytes = (std::max<size_t>(bytes, 1) + 255) & ~(size_t)255;
        auto it = free_.lower_bound(bytes);
        if (it != free_.end() && it->first <= 2 * bytes + ((size_t)1 << 20)) {
            *p = it->second;
            free_.erase(it);
            return cudaSuccess;
        }
        cudaError_t e = cudaMalloc(p, bytes);
        if (e == cudaErrorMemoryAllocation) {
            cudaGetLastError();
            release();
            e = cudaMalloc(p, bytes);
        }
        if (e == cudaSuccess) sizes_[*p] = bytes;
        return e;
    }
    void free(void* p) {
        if (!p) return;
        auto it = sizes_.find(p);
        if (it == sizes_.end()) return;
        free_.emplace(it->second, p);
    }
    void release() {
        for (auto& kv : free_) {
            cudaFree(kv.second);
            sizes_.erase(kv.second);
        }
        free_.clear();
    }
};

struct DevPlanStore {
    HostPlan host;
    DevPlan dev{};
    void* mem = nullptr;
};

}  // namespace

namespace tcu {
thread_local Profiler* g_prof = nullptr;
thread_local DeviceAllocator* g_call_pool = nullptr;
void set_error_message(const char* msg) { g_last_error = msg; }
}

struct tcu_context {
    Profiler prof;
    DevicePool pool;
    int device = 0;
    cudaStream_t stream = nullptr;
    std::recursive_mutex mu;
    std::map<int, std::unique_ptr<DevPlanStore>> plans;
    long long launches = 0;
    double* d_partial = nullptr;  // reduction scratch (8 * 256 doubles)
    cplx* d_cpartial = nullptr;   // complex reduction scratch (64 * 256)
    double* d_small = nullptr;    // 64 doubles
    cplx* d_csmall = nullptr;     // 64 complex
    int* d_status = nullptr;
    double* d_lfac = nullptr;     // sqrt((l-m)!/(l+m)!) table up to degree 16
    // GMRES preconditioner settings (tcu_context_set_learned_weights)
    double precond_reach = -1.0;  // near-field reach in sphere diameters (< 0: the compiled-in one)
    std::vector<double> learned_weights;  // empty: the compiled-in weights
    long long fallbacks = 0;      // mixed solves finished by a second factor
    std::set<tcu_factor*> factors;  // live factors (destroyed with the context)
    double refine_target = 1e-13; // refinement stops at ||r|| <= refine_target ||T b||
    double fallback_above = 1e-12;  // mixed solves left above this finish in FP64
    size_t auto_crossover = 2048;   // TCU_AUTO: mixed from this many unknowns on (tcu_context_autotune)
    std::vector<tcu_context*> workers;  // batched solves: a context (stream, scratch, pool) per host worker
    int panel_rows = 0;  // least rows per LU panel CTA (0: the default); batch workers take 192
};

struct tcu_factor {
    tcu_context* ctx = nullptr;
    int L = 0, N = 0;
    size_t n = 0;
    int precision = 0;
    double k0 = 0;
    double* d_pos = nullptr;
    double* d_radii = nullptr;
    cplx* d_eps = nullptr;
    cplx* d_T = nullptr;
    void* d_A = nullptr;
    double2* d_inv = nullptr;  // inverses of the diagonal blocks of L and U
    LuWork wk;
    double* d_scale = nullptr;       // row scales (n) then column scales (n) when equilibrated
    cplx* d_Z = nullptr;             // stored pair tables of the refinement's FP64 residual (lmax 2..5)
    bool scaled = false;
    tcu_factor* fallback = nullptr;  // FP64 factor of a mixed factor whose refinement stalled
    unsigned sweep_epoch = 0;        // epochs of the persistent triangular sweeps
};

namespace {

struct ProfGuard {
    Profiler* prev;
    explicit ProfGuard(tcu_context* ctx) : prev(g_prof) { g_prof = &ctx->prof; }
    ~ProfGuard() { g_prof = prev; }
};

tcu_status cuda_check(cudaError_t e, const char* what) {
    if (e == cudaSuccess) return TCU_OK;
    if (e == cudaErrorMemoryAllocation) return fail(TCU_OUT_OF_MEMORY, std::string(what) + ": " + cudaGetErrorString(e));
    return fail(TCU_DEVICE_ERROR, std::string(what) + ": " + cudaGetErrorString(e));
}
#define CK(call, what)                              \
    do {                                            \
        tcu_status _s = cuda_check((call), (what)); \
        if (_s != TCU_OK) return _s;                \
    } while (0)

bool finite_all(const double* p, size_t n) {
    for (size_t i = 0; i < n; ++i)
        if (!std::isfinite(p[i])) return false;
    return true;
}

// cluster/spheres.rs:99-133
tcu_status validate_spheres(int L, double k0, size_t N, const double* radii, const double* eps, const double* pos) {
    if (L < 1 || L > 10) return fail(TCU_INVALID_INPUT, "require 1 <= lmax <= 10");
    if (!std::isfinite(k0) || k0 <= 0.0 || N == 0 || !radii || !eps || !pos)
        return fail(TCU_INVALID_INPUT,
                    "require positive finite k0 and radii, and matching finite permittivities and positions");
    for (size_t i = 0; i < N; ++i)
        if (!std::isfinite(radii[i]) || radii[i] <= 0.0)
            return fail(TCU_INVALID_INPUT,
                        "require positive finite k0 and radii, and matching finite permittivities and positions");
    if (!finite_all(eps, 2 * N) || !finite_all(pos, 3 * N))
        return fail(TCU_INVALID_INPUT,
                    "require positive finite k0 and radii, and matching finite permittivities and positions");
    // Touching or overlapping pairs are closer than 2 max(radius): bin the centres into cubic
    // cells of that edge and test each sphere against the spheres of its own and the 13
    // preceding neighbour cells (every pair once), which finds the same pairs as testing all
    // N^2 / 2 of them.
    double rmax = 0.0, lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
    for (size_t i = 0; i < N; ++i) {
        rmax = std::max(rmax, radii[i]);
        for (int a = 0; a < 3; ++a) {
            lo[a] = std::min(lo[a], pos[3 * i + a]);
            hi[a] = std::max(hi[a], pos[3 * i + a]);
        }
    }
    const double edge = 2.0 * rmax;
    long dims[3];
    for (int a = 0; a < 3; ++a) {
        const double span = (hi[a] - lo[a]) / edge;
        if (!std::isfinite(span) || span > 4.0e6)
            return fail(TCU_INVALID_INPUT,
                        "spherical particles must have finite separation and must not touch or overlap");
        dims[a] = (long)span + 1;
    }
    auto cell = [&](size_t i, int a) { return std::min(dims[a] - 1, (long)((pos[3 * i + a] - lo[a]) / edge)); };
    std::vector<std::pair<long long, size_t>> order(N);
    for (size_t i = 0; i < N; ++i)
        order[i] = {((long long)cell(i, 0) * dims[1] + cell(i, 1)) * dims[2] + cell(i, 2), i};
    std::sort(order.begin(), order.end());
    auto touching = [&](size_t i, size_t j) {
        const double d = std::hypot(std::hypot(pos[3 * i] - pos[3 * j], pos[3 * i + 1] - pos[3 * j + 1]),
                                    pos[3 * i + 2] - pos[3 * j + 2]);
        return d <= radii[i] + radii[j] || !std::isfinite(d);
    };
    for (size_t q = 0; q < N; ++q) {
        const size_t i = order[q].second;
        const long cx = cell(i, 0), cy = cell(i, 1), cz = cell(i, 2);
        for (long dx = -1; dx <= 1; ++dx)
            for (long dy = -1; dy <= 1; ++dy)
                for (long dz = -1; dz <= 1; ++dz) {
                    const long x = cx + dx, y = cy + dy, z = cz + dz;
                    if (x < 0 || y < 0 || z < 0 || x >= dims[0] || y >= dims[1] || z >= dims[2]) continue;
                    const long long key = ((long long)x * dims[1] + y) * dims[2] + z;
                    auto it = std::lower_bound(order.begin(), order.end(), std::make_pair(key, (size_t)0));
                    for (; it != order.end() && it->first == key; ++it)
                        if (it->second < i && touching(i, it->second))
                            return fail(TCU_INVALID_INPUT,
                                        "spherical particles must have finite separation and must not touch or "
                                        "overlap");
                }
    }
    return TCU_OK;
}

tcu_status get_plan(tcu_context* ctx, int L, const DevPlan** out) {
    auto it = ctx->plans.find(L);
    if (it == ctx->plans.end()) {
        auto store = std::make_unique<DevPlanStore>();
        store->host = build_plan(L);
        HostPlan& h = store->host;
        size_t ncombo = (size_t)h.nlm * h.nlm;
        size_t nterm = h.idx.size();
        // every array starts on a 256-byte boundary (the weights are read as 16-byte double2)
        auto up = [](size_t v) { return (v + 255) & ~(size_t)255; };
        size_t off_combo = 0, off_w = up(ncombo * 8), off_refl = up(off_w + nterm * 16),
               off_idx = up(off_refl + h.reflection.size() * 8);
        size_t total = off_idx + nterm * 2 + 16;
        CK(cudaMalloc(&store->mem, total), "plan allocation");
        char* base = (char*)store->mem;
        CK(cudaMemcpy(base + off_combo, h.combo.data(), ncombo * 8, cudaMemcpyHostToDevice), "plan upload");
        CK(cudaMemcpy(base + off_w, h.w.data(), nterm * 16, cudaMemcpyHostToDevice), "plan upload");
        CK(cudaMemcpy(base + off_refl, h.reflection.data(), h.reflection.size() * 8, cudaMemcpyHostToDevice),
           "plan upload");
        CK(cudaMemcpy(base + off_idx, h.idx.data(), nterm * 2, cudaMemcpyHostToDevice), "plan upload");
        DevPlan& d = store->dev;
        d.L = L;
        d.nlm = h.nlm;
        d.order = h.order;
        d.tsize = (h.order + 1) * (h.order + 1);
        d.combo = (const int2*)(base + off_combo);
        d.w = (const double2*)(base + off_w);
        d.reflection = (const double*)(base + off_refl);
        d.idx = (const uint16_t*)(base + off_idx);
        it = ctx->plans.emplace(L, std::move(store)).first;
    }
    *out = &it->second->dev;
    return TCU_OK;
}

tcu_status sync_status(tcu_context* ctx, const char* what) {
    cudaError_t e = cudaStreamSynchronize(ctx->stream);
    if (e == cudaSuccess) e = cudaGetLastError();
    return cuda_check(e, what);
}

tcu_status read_status(tcu_context* ctx, const char* what) {
    int st = 0;
    CK(cudaMemcpyAsync(&st, ctx->d_status, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream), what);
    tcu_status s = sync_status(ctx, what);
    if (s != TCU_OK) return s;
    if (st == 5) return fail(TCU_SINGULAR, std::string(what) + ": numerically singular");
    if (st == 8) return fail(TCU_TIMEOUT, std::string(what) + ": a device-side wait gave up");
    if (st != 0) return fail(TCU_DEVICE_ERROR, std::string(what) + ": device status " + std::to_string(st));
    return TCU_OK;
}

template <typename T>
tcu_status dev_alloc(tcu_context* ctx, T** p, size_t count, const char* what) {
    return cuda_check(ctx->pool.alloc((void**)p, std::max<size_t>(count, 1) * sizeof(T)), what);
}

// A per-call device buffer from the context pool.
struct DevBuf {
    tcu_context* ctx;
    void* p = nullptr;
    explicit DevBuf(tcu_context* c) : ctx(c) {}
    cudaError_t alloc(size_t bytes) { return ctx->pool.alloc(&p, bytes); }
    ~DevBuf() {
        if (p) ctx->pool.free(p);
    }
};

// Sub-buffers of one allocation, each on a 256-byte boundary.
struct Arena {
    std::vector<size_t> offs;
    size_t total = 0;
    size_t add(size_t bytes) {
        size_t o = total;
        offs.push_back(o);
        total = (total + bytes + 255) & ~(size_t)255;
        return o;
    }
    template <typename T>
    T* at(void* base, size_t off) const {
        return (T*)((char*)base + off);
    }
};

// The y = zadd + alpha x + beta T C x operator in chunks of at most 8 columns.
void apply_op(tcu_context* ctx, const DevPlan* P, int N, double k0, const double* d_pos, const cplx* d_T, const cplx* x,
              size_t n, int ncol, const cplx* zadd, double alpha, double beta, bool singular, cplx* y) {
    for (int c0 = 0; c0 < ncol; c0 += 8) {
        int nc = std::min(8, ncol - c0);
        launch_apply(*P, N, k0, d_pos, d_T, x + c0 * n, n, nc, zadd ? zadd + c0 * n : nullptr, alpha, beta, singular,
                     y + c0 * n, ctx->stream);
        ++ctx->launches;
    }
}

tcu_status factor_impl(tcu_context* ctx, int L, double k0, size_t N, const double* radii_h, const double* eps_h,
                       const double* pos_h, const double* radii_d, const double* eps_d, const double* pos_d,
                       int precision, tcu_factor** out, bool reduced = true) {
    if (!out) return fail(TCU_INVALID_INPUT, "null output handle");
    *out = nullptr;
    if (precision != TCU_FP64 && precision != TCU_MIXED) return fail(TCU_INVALID_INPUT, "unknown precision");
    tcu_status s = validate_spheres(L, k0, N, radii_h, eps_h, pos_h);
    if (s) return s;
    const DevPlan* P;
    s = get_plan(ctx, L, &P);
    if (s) return s;
    size_t M = 2 * (size_t)L * (L + 2);
    size_t n = N * M;
    if (n > 28416) return fail(TCU_INVALID_INPUT, "dense cluster dimension above 28416; use the iterative solver");
    auto f = std::make_unique<tcu_factor>();
    f->ctx = ctx;
    f->L = L;
    f->N = (int)N;
    f->n = n;
    f->precision = precision;
    f->k0 = k0;
    // reduced: the piece formats the environment may ask for (FP16 pieces, two-pass TF32);
    // the refinement's fallback factor takes the three-pass TF32 split instead
    f->wk.f16_pieces = reduced && split_f16_default();
    f->wk.two_pass = reduced && !f->wk.f16_pieces && split_two_pass_default();
    f->wk.panel_rows = ctx->panel_rows;
    auto cleanup = [&]() {
        for (void* q : {(void*)f->d_pos, (void*)f->d_radii, (void*)f->d_eps, (void*)f->d_T, f->d_A,
                        (void*)f->d_inv, (void*)f->wk.piv, f->wk.pack, (void*)f->d_scale, (void*)f->d_Z})
            ctx->pool.free(q);
    };
    tcu_status e = TCU_OK;
    do {
        if ((e = dev_alloc(ctx, &f->d_pos, 3 * N, "positions"))) break;
        if ((e = dev_alloc(ctx, &f->d_radii, N, "radii"))) break;
        if ((e = dev_alloc(ctx, &f->d_eps, N, "permittivities"))) break;
        if ((e = dev_alloc(ctx, &f->d_T, N * L * 4, "T blocks"))) break;
        cudaMemcpyKind kind = pos_d ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
        if ((e = cuda_check(cudaMemcpyAsync(f->d_pos, pos_d ? pos_d : pos_h, 3 * N * 8, kind, ctx->stream), "copy"))) break;
        if ((e = cuda_check(cudaMemcpyAsync(f->d_radii, radii_d ? radii_d : radii_h, N * 8, kind, ctx->stream), "copy")))
            break;
        if ((e = cuda_check(cudaMemcpyAsync(f->d_eps, eps_d ? eps_d : eps_h, N * 16, kind, ctx->stream), "copy"))) break;
        size_t elem = precision == TCU_FP64 ? 16 : 8;
        if ((e = cuda_check(ctx->pool.alloc(&f->d_A, n * n * elem), "interaction matrix"))) break;
        if (precision == TCU_MIXED && tf32_enabled()) {
            f->wk.pack_bytes = tf32_pack_bytes((int)n);
            if ((e = cuda_check(ctx->pool.alloc(&f->wk.pack, f->wk.pack_bytes), "tensor-core operands"))) break;
        }
        size_t ws = lu_workspace_bytes((int)n, precision == TCU_MIXED);
        void* wmem = nullptr;
        if ((e = cuda_check(ctx->pool.alloc(&wmem, ws), "LU workspace"))) break;
        f->wk.piv = (int*)wmem;
        f->wk.perm = f->wk.piv + n;
        f->wk.barrier = (unsigned*)(f->wk.perm + n);
        f->wk.status = (int*)(f->wk.barrier + 4);
        f->wk.cand = (void*)(((uintptr_t)(f->wk.status + 4) + 255) & ~(uintptr_t)255);
        CK(cudaMemsetAsync(ctx->d_status, 0, sizeof(int), ctx->stream), "status");
        CK(cudaMemsetAsync(f->wk.status, 0, sizeof(int), ctx->stream), "status");
        launch_mie(L, k0, (int)N, f->d_radii, f->d_eps, f->d_T, ctx->d_status, ctx->stream);
        ++ctx->launches;
        if ((e = read_status(ctx, "Mie coefficients"))) break;
        launch_assemble(*P, (int)N, k0, f->d_pos, f->d_T, f->d_A, n, precision == TCU_MIXED, ctx->stream);
        ++ctx->launches;
        if (apply_gemm_supported(*P) && stored_tables_enabled()) {
            // the refinement's residuals apply the FP64 operator from stored pair tables (at most a
            // fifth of the matrix's bytes); without room they rebuild the tables per application
            void* z = nullptr;
            if (ctx->pool.alloc(&z, stored_tables_bytes(*P, (int)N, STORED_FULL)) == cudaSuccess) {
                f->d_Z = (cplx*)z;
                build_stored_tables(*P, (int)N, k0, f->d_pos, STORED_FULL, f->d_Z, ctx->stream);
                ++ctx->launches;
            } else {
                cudaGetLastError();
            }
        }
        {
            // equilibrate when an entry exceeds 10 (then the unit diagonal no longer bounds the
            // spread; linalg/mod.rs:137-228)
            if ((e = dev_alloc(ctx, &f->d_scale, 2 * n, "scales"))) break;
            DevBuf eq(ctx);
            if ((e = cuda_check(eq.alloc(equilibrate_scratch_doubles((int)n) * sizeof(double)), "scales"))) break;
            if ((e = equilibrate(f->d_A, precision == TCU_MIXED, (int)n, 10.0, f->d_scale, f->d_scale + n,
                                 (double*)eq.p, &f->scaled, ctx->stream, &ctx->launches))) {
                e = fail(e, "equilibration failed");
                break;
            }
        }
        int rc;
        if (precision == TCU_FP64)
            rc = lu_factor_fp64((double2*)f->d_A, (int)n, f->wk, ctx->stream, &ctx->launches);
        else
            rc = lu_factor_fp32((float2*)f->d_A, (int)n, f->wk, ctx->stream, &ctx->launches, tf32_enabled());
        if (rc) {
            e = fail(TCU_DEVICE_ERROR, "LU panel launch failed (cooperative launch or shared memory)");
            break;
        }
        int st = 0;
        if ((e = cuda_check(cudaMemcpyAsync(&st, f->wk.status, 4, cudaMemcpyDeviceToHost, ctx->stream), "LU"))) break;
        if ((e = sync_status(ctx, "LU factorization"))) break;
        if (st == 5) {
            e = fail(TCU_SINGULAR, "LU factorization: zero pivot");
            break;
        }
        if (st == 8) {
            e = fail(TCU_TIMEOUT, "LU factorization: a device-side wait gave up");
            break;
        }
        if (st == 6) {
            e = fail(TCU_OUT_OF_MEMORY, "LU factorization: no memory for the packed tensor-core operands");
            break;
        }
        if (st != 0) {
            e = fail(TCU_DEVICE_ERROR, "LU factorization: device status " + std::to_string(st));
            break;
        }
        if ((e = cuda_check(ctx->pool.alloc((void**)&f->d_inv, lu_inverse_bytes((int)n)), "block inverses"))) break;
        if (precision == TCU_FP64)
            lu_block_inverses_fp64((const double2*)f->d_A, (int)n, f->d_inv, ctx->stream, &ctx->launches);
        else
            lu_block_inverses_fp32((const float2*)f->d_A, (int)n, f->d_inv, ctx->stream, &ctx->launches);
        if ((e = sync_status(ctx, "block inverses"))) break;
    } while (0);
    if (e) {
        cleanup();
        return e;
    }
    *out = f.release();
    ctx->factors.insert(*out);
    return TCU_OK;
}

tcu_status solve_impl(tcu_factor* f, const double* B, int p, double* X, tcu_certificate* certs, bool device) {
    if (!f || !B || !X || p <= 0) return fail(TCU_INVALID_INPUT, "require a factor and at least one column");
    if (p > 8) {  // the norms of a context reduce at most 8 columns at once
        for (int c0 = 0; c0 < p; c0 += 8) {
            const size_t off = 2 * f->n * (size_t)c0;
            tcu_status s = solve_impl(f, B + off, std::min(8, p - c0), X + off, certs ? certs + c0 : nullptr, device);
            if (s) return s;
        }
        return TCU_OK;
    }
    tcu_context* ctx = f->ctx;
    std::lock_guard<std::recursive_mutex> lock(ctx->mu);
    ProfGuard pg(ctx);
    CK(cudaSetDevice(ctx->device), "device");
    const DevPlan* P;
    tcu_status s = get_plan(ctx, f->L, &P);
    if (s) return s;
    size_t n = f->n;
    if (!device && !finite_all(B, 2 * n * p))
        return fail(TCU_INVALID_INPUT,
                    "require finite channel-by-illumination columns matching the factorization");
    DevBuf bufs(ctx);
    size_t per = n * p;
    const size_t xf_bytes = f->d_Z ? stored_inputs_bytes(*P, f->N, STORED_FULL, p) : 0;
    CK(bufs.alloc(6 * per * sizeof(cplx) + xf_bytes), "solve buffers");
    cplx* b = (cplx*)bufs.p;
    cplx* tb = b + per;
    cplx* x = tb + per;
    cplx* r = x + per;
    cplx* tmp = r + per;  // 2 per
    cplx* xf = tmp + 2 * per;  // packed inputs of the stored-table residual
    CK(cudaMemcpyAsync(b, B, per * 16, device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, ctx->stream),
       "copy rhs");
    launch_apply_t(f->L, f->N, f->d_T, b, p, tb, ctx->stream);
    ++ctx->launches;
    std::vector<double> rn(p), bn(p);
    vec_norms(tb, n, p, ctx->d_small, ctx->d_partial, ctx->stream);
    ctx->launches += 2;
    CK(cudaMemcpyAsync(bn.data(), ctx->d_small, p * 8, cudaMemcpyDeviceToHost, ctx->stream), "norms");
    int sweeps = 0;
    auto lu_apply = [&](cplx* v) {
        if (f->scaled) scale_rows(v, f->d_scale, n, p, ctx->stream);  // R v
        if (f->precision == TCU_FP64)
            lu_solve_fp64((const double2*)f->d_A, (int)n, f->wk.perm, f->d_inv, v, tmp, p, ctx->stream,
                          &ctx->launches, &f->sweep_epoch, f->wk.status);
        else
            lu_solve_fp32((const float2*)f->d_A, (int)n, f->wk.perm, f->d_inv, v, tmp, p, ctx->stream,
                          &ctx->launches, &f->sweep_epoch, f->wk.status);
        if (f->scaled) {
            scale_rows(v, f->d_scale + n, n, p, ctx->stream);  // C (A')^-1 R v
            ctx->launches += 2;
        }
    };
    int sweep_status = 0;
    auto residual = [&]() -> tcu_status {
        // r = T b - (x - T C x)
        if (f->d_Z) {
            launch_apply_stored(*P, f->N, STORED_FULL, f->d_Z, f->d_T, x, n, p, tb, -1.0, 1.0, r, xf, f->wk.status,
                                ctx->stream);
            ctx->launches += 2;
        } else {
            apply_op(ctx, P, f->N, f->k0, f->d_pos, f->d_T, x, n, p, tb, -1.0, 1.0, true, r);
        }
        vec_norms(r, n, p, ctx->d_small, ctx->d_partial, ctx->stream);
        ctx->launches += 2;
        CK(cudaMemcpyAsync(rn.data(), ctx->d_small, p * 8, cudaMemcpyDeviceToHost, ctx->stream), "norms");
        CK(cudaMemcpyAsync(&sweep_status, f->wk.status, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream), "status");
        tcu_status s2 = sync_status(ctx, "residual");
        if (s2) return s2;
        if (sweep_status == 8) return fail(TCU_TIMEOUT, "refinement: a device-side wait gave up");
        return TCU_OK;
    };
    CK(cudaMemcpyAsync(x, tb, per * 16, cudaMemcpyDeviceToDevice, ctx->stream), "copy");
    lu_apply(x);
    sweeps = 1;
    if ((s = residual())) return s;
    {
        // iterative refinement in FP64: up to 10 sweeps on mixed factors (20 with two-pass updates), 2 on
        // FP64 factors
        const double tol = ctx->refine_target;
        double prev = INFINITY;
        const int max_sweeps = f->precision == TCU_MIXED ? (f->wk.two_pass ? 20 : 10) : 2;
        for (int it = 0; it < max_sweeps; ++it) {
            double worst = 0.0;
            for (int c = 0; c < p; ++c) worst = std::max(worst, bn[c] > 0 ? rn[c] / bn[c] : rn[c]);
            if (worst <= tol || !(worst < 0.5 * prev)) break;
            prev = worst;
            lu_apply(r);
            vec_axpy(x, r, n, p, ctx->stream);
            ++ctx->launches;
            ++sweeps;
            if ((s = residual())) return s;
        }
    }
    if (f->precision == TCU_MIXED) {
        // refinement stalled above the FP64 target (an ill-scaled operator beyond the reach of
        // the TF32 factors): finish with an FP64 factor of the same cluster, kept for later solves
        double worst = 0.0;
        for (int c = 0; c < p; ++c) worst = std::max(worst, bn[c] > 0 ? rn[c] / bn[c] : rn[c]);
        if (!(worst <= ctx->fallback_above)) {
            // FP16 pieces first fall back to a mixed factor with TF32 pieces (which keep 22
            // bits relative to every element), that one in turn to FP64
            if (!f->fallback) {
                std::vector<double> hr(f->N), he(2 * (size_t)f->N), hp(3 * (size_t)f->N);
                CK(cudaMemcpyAsync(hr.data(), f->d_radii, f->N * 8, cudaMemcpyDeviceToHost, ctx->stream), "copy");
                CK(cudaMemcpyAsync(he.data(), f->d_eps, f->N * 16, cudaMemcpyDeviceToHost, ctx->stream), "copy");
                CK(cudaMemcpyAsync(hp.data(), f->d_pos, f->N * 24, cudaMemcpyDeviceToHost, ctx->stream), "copy");
                if ((s = sync_status(ctx, "fallback"))) return s;
                const bool to_tf32 = f->wk.f16_pieces || f->wk.two_pass;
                if ((s = factor_impl(ctx, f->L, f->k0, f->N, hr.data(), he.data(), hp.data(), nullptr, nullptr,
                                     nullptr, to_tf32 ? TCU_MIXED : TCU_FP64, &f->fallback, false)))
                    return s;
            }
            ++ctx->fallbacks;
            return solve_impl(f->fallback, B, p, X, certs, device);
        }
    }
    for (int c = 0; c < p; ++c)
        if (!std::isfinite(rn[c])) return fail(TCU_SINGULAR, "non-finite solution: numerically singular operator");
    CK(cudaMemcpyAsync(X, x, per * 16, device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost, ctx->stream),
       "copy solution");
    if ((s = sync_status(ctx, "solve"))) return s;
    if (certs)
        for (int c = 0; c < p; ++c) {
            certs[c].iterations = sweeps;
            certs[c].residual_norm = rn[c];
            certs[c].rhs_norm = bn[c];
        }
    return TCU_OK;
}

// Adjoint solve Y = (I - T C)^-H G with a factor (cluster/interaction.rs:221-227 uses it for
// pullback_incident; linalg/mod.rs:436 solve_adjoint_in_place): A^-H g = R P^T L^-H U^-H C g with
// the scales R, C of the factor, refined in FP64 against the matrix-free adjoint operator like
// the forward solve. th: return T^H Y instead (the incident-field gradient).
tcu_status solve_adjoint_impl(tcu_factor* f, const double* G, int p, double* Y, tcu_certificate* certs, bool th) {
    if (!f || !G || !Y || p <= 0) return fail(TCU_INVALID_INPUT, "require a factor and at least one column");
    if (p > 8) {  // the norms of a context reduce at most 8 columns at once
        for (int c0 = 0; c0 < p; c0 += 8) {
            const size_t off = 2 * f->n * (size_t)c0;
            tcu_status s =
                solve_adjoint_impl(f, G + off, std::min(8, p - c0), Y + off, certs ? certs + c0 : nullptr, th);
            if (s) return s;
        }
        return TCU_OK;
    }
    tcu_context* ctx = f->ctx;
    std::lock_guard<std::recursive_mutex> lock(ctx->mu);
    ProfGuard pg(ctx);
    CK(cudaSetDevice(ctx->device), "device");
    const DevPlan* P;
    tcu_status s = get_plan(ctx, f->L, &P);
    if (s) return s;
    const size_t n = f->n, per = n * p;
    if (!finite_all(G, 2 * per))
        return fail(TCU_INVALID_INPUT, "require finite channel-by-illumination columns matching the factorization");
    DevBuf bufs(ctx);
    const size_t tmpc = adjoint_solve_tmp((int)n, p);
    const size_t xfc = f->d_Z ? stored_inputs_bytes(*P, f->N, STORED_FULL, p) / sizeof(cplx) : 0;
    CK(bufs.alloc((5 * per + tmpc + xfc) * sizeof(cplx)), "adjoint solve buffers");
    cplx* g = (cplx*)bufs.p;
    cplx* y = g + per;
    cplx* r = y + per;
    cplx* t1 = r + per;
    cplx* t2 = t1 + per;
    cplx* xf = t2 + per;  // packed inputs of the stored-table coupling product
    cplx* tmp = xf + xfc;
    CK(cudaMemsetAsync(ctx->d_status, 0, 4, ctx->stream), "status");
    CK(cudaMemcpyAsync(g, G, per * 16, cudaMemcpyHostToDevice, ctx->stream), "copy rhs");
    std::vector<double> rn(p), bn(p);
    vec_norms(g, n, p, ctx->d_small, ctx->d_partial, ctx->stream);
    CK(cudaMemcpyAsync(bn.data(), ctx->d_small, p * 8, cudaMemcpyDeviceToHost, ctx->stream), "norms");
    auto lu_adjoint = [&](cplx* v) {
        if (f->scaled) scale_rows(v, f->d_scale + n, n, p, ctx->stream);  // C g
        if (f->precision == TCU_FP64)
            lu_solve_adjoint_fp64((const double2*)f->d_A, (int)n, f->wk.perm, f->d_inv, v, tmp, p, ctx->stream,
                                  &ctx->launches);
        else
            lu_solve_adjoint_fp32((const float2*)f->d_A, (int)n, f->wk.perm, f->d_inv, v, tmp, p, ctx->stream,
                                  &ctx->launches);
        if (f->scaled) scale_rows(v, f->d_scale, n, p, ctx->stream);  // R
    };
    auto residual = [&]() -> tcu_status {  // r = g - A^H y
        launch_apply_adjoint(*P, f->N, f->k0, f->d_pos, f->d_T, y, n, p, r, t1, t2, ctx->stream, &ctx->launches,
                             f->d_Z, xf, ctx->d_status);
        vec_sub(r, g, r, n, p, ctx->stream);
        vec_norms(r, n, p, ctx->d_small, ctx->d_partial, ctx->stream);
        ctx->launches += 3;
        CK(cudaMemcpyAsync(rn.data(), ctx->d_small, p * 8, cudaMemcpyDeviceToHost, ctx->stream), "norms");
        return read_status(ctx, "adjoint residual");
    };
    CK(cudaMemcpyAsync(y, g, per * 16, cudaMemcpyDeviceToDevice, ctx->stream), "copy");
    lu_adjoint(y);
    int sweeps = 1;
    if ((s = residual())) return s;
    const double tol = ctx->refine_target;
    double prev = INFINITY;
    const int max_sweeps = f->precision == TCU_MIXED ? (f->wk.two_pass ? 20 : 10) : 2;
    auto worst_of = [&]() {
        double w = 0.0;
        for (int c = 0; c < p; ++c) w = std::max(w, bn[c] > 0 ? rn[c] / bn[c] : rn[c]);
        return w;
    };
    for (int it = 0; it < max_sweeps; ++it) {
        const double worst = worst_of();
        if (worst <= tol || !(worst < 0.5 * prev)) break;
        prev = worst;
        lu_adjoint(r);
        vec_axpy(y, r, n, p, ctx->stream);
        ++ctx->launches;
        ++sweeps;
        if ((s = residual())) return s;
    }
    if (f->precision == TCU_MIXED && !(worst_of() <= ctx->fallback_above)) {
        if (!f->fallback) {
            std::vector<double> hr(f->N), he(2 * (size_t)f->N), hp(3 * (size_t)f->N);
            CK(cudaMemcpyAsync(hr.data(), f->d_radii, f->N * 8, cudaMemcpyDeviceToHost, ctx->stream), "copy");
            CK(cudaMemcpyAsync(he.data(), f->d_eps, f->N * 16, cudaMemcpyDeviceToHost, ctx->stream), "copy");
            CK(cudaMemcpyAsync(hp.data(), f->d_pos, f->N * 24, cudaMemcpyDeviceToHost, ctx->stream), "copy");
            if ((s = sync_status(ctx, "fallback"))) return s;
            const bool to_tf32 = f->wk.f16_pieces || f->wk.two_pass;
            if ((s = factor_impl(ctx, f->L, f->k0, f->N, hr.data(), he.data(), hp.data(), nullptr, nullptr, nullptr,
                                 to_tf32 ? TCU_MIXED : TCU_FP64, &f->fallback, false)))
                return s;
        }
        ++ctx->fallbacks;
        return solve_adjoint_impl(f->fallback, G, p, Y, certs, th);
    }
    for (int c = 0; c < p; ++c)
        if (!std::isfinite(rn[c])) return fail(TCU_SINGULAR, "non-finite solution: numerically singular operator");
    if (th) {
        launch_apply_th(f->L, f->N, f->d_T, y, n, p, r, ctx->stream);
        ++ctx->launches;
    }
    CK(cudaMemcpyAsync(Y, th ? r : y, per * 16, cudaMemcpyDeviceToHost, ctx->stream), "copy solution");
    if ((s = sync_status(ctx, "adjoint solve"))) return s;
    if (certs)
        for (int c = 0; c < p; ++c) {
            certs[c].iterations = sweeps;
            certs[c].residual_norm = rn[c];
            certs[c].rhs_norm = bn[c];
        }
    return TCU_OK;
}

// A factor applied once (no refinement): v <- A^-1 v with the row/column scales; the coarse
// solve of the two-level preconditioners. Owns the factor.
struct FactorCoarse : CoarseSolve {
    tcu_factor* f = nullptr;
    cplx* tmp = nullptr;
    ~FactorCoarse() override {
        if (tmp) f->ctx->pool.free(tmp);
        if (f) tcu_factor_destroy(f);
    }
    tcu_status solve(double2* v, cudaStream_t st) override {
        tcu_context* ctx = f->ctx;
        const size_t n = f->n;
        if (f->scaled) scale_rows(v, f->d_scale, n, 1, st);
        if (f->precision == TCU_FP64)
            lu_solve_fp64((const double2*)f->d_A, (int)n, f->wk.perm, f->d_inv, v, tmp, 1, st, &ctx->launches,
                          &f->sweep_epoch, f->wk.status);
        else
            lu_solve_fp32((const float2*)f->d_A, (int)n, f->wk.perm, f->d_inv, v, tmp, 1, st, &ctx->launches,
                          &f->sweep_epoch, f->wk.status);
        if (f->scaled) scale_rows(v, f->d_scale + n, n, 1, st);
        return TCU_OK;
    }
};

// Host worker threads of tcu_batch_solve: TCU_BATCH_WORKERS (1..8), default 4.
int batch_workers() {
    const char* e = getenv("TCU_BATCH_WORKERS");
    const int v = e ? atoi(e) : 4;
    return std::max(1, std::min(8, v));
}

// The stored-table operator for the applications of GMRES: lmax 2..5 in product form, unless
// TCU_APPLY is "fly" or "terms", and only while the tables take at most half of the free device
// memory (and at most 64 GB).
bool use_stored_tables(const DevPlan& P, int N) {
    if (!apply_gemm_supported(P) || !stored_tables_enabled()) return false;
    const size_t bytes = stored_tables_bytes(P, N, STORED_FULL);
    if (bytes == 0 || bytes > ((size_t)64 << 30)) return false;
    size_t fr = 0, tot = 0;
    if (cudaMemGetInfo(&fr, &tot) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return bytes <= fr / 2;
}

// The dipole (lmax 1) system of a cluster: factored (complex64 from 2048 modes on, else FP64) up
// to 6144 dipole modes; above, no factor is made (out stays empty) and the two-level
// preconditioner solves the dipole system by an inner GMRES on its matrix-free dipole block.
constexpr size_t COARSE_LU_MAX = 6144;
tcu_status make_coarse(tcu_context* ctx, double k0, size_t N, const double* radii, const double* eps,
                       const double* pos, std::unique_ptr<CoarseSolve>* out, bool factor_always = false) {
    if (6 * N > COARSE_LU_MAX && !factor_always) return TCU_OK;
    auto c = std::make_unique<FactorCoarse>();
    const int prec = 6 * N >= 2048 ? TCU_MIXED : TCU_FP64;
    tcu_status s = factor_impl(ctx, 1, k0, N, radii, eps, pos, nullptr, nullptr, nullptr, prec, &c->f);
    if (s) return s;
    if ((s = dev_alloc(ctx, &c->tmp, 2 * 6 * N, "coarse solve buffers"))) return s;
    *out = std::move(c);
    return TCU_OK;
}

}  // namespace

// =========================================================================================
extern "C" {

const char* tcu_last_error_message(void) { return g_last_error.c_str(); }

tcu_status tcu_context_create(int device, tcu_context** out) {
    if (!out) return fail(TCU_INVALID_INPUT, "null output handle");
    *out = nullptr;
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0)
        return fail(TCU_DEVICE_ERROR, "no CUDA device available: the library has no CPU path");
    if (device < 0 || device >= count) return fail(TCU_INVALID_INPUT, "device index out of range");
    CK(cudaSetDevice(device), "set device");
    cudaDeviceProp prop;
    CK(cudaGetDeviceProperties(&prop, device), "device properties");
    if (prop.major != 10) return fail(TCU_DEVICE_ERROR, "the library is built for sm_100a (B200) only");
    auto ctx = std::make_unique<tcu_context>();
    ctx->device = device;
    CK(cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking), "stream");
    CK(cudaMalloc(&ctx->d_partial, 8 * 256 * sizeof(double)), "scratch");
    CK(cudaMalloc(&ctx->d_cpartial, 64 * 256 * sizeof(cplx)), "scratch");
    CK(cudaMalloc(&ctx->d_small, 64 * sizeof(double)), "scratch");
    CK(cudaMalloc(&ctx->d_csmall, 64 * sizeof(cplx)), "scratch");
    CK(cudaMalloc(&ctx->d_status, 16), "scratch");
    std::vector<double> lfac(17 * 17);
    for (int l = 0; l <= 16; ++l)
        for (int m = -l; m <= l; ++m)
            lfac[l * l + l + m] = std::exp(0.5 * (std::lgamma(l - m + 1.0) - std::lgamma(l + m + 1.0)));
    CK(cudaMalloc(&ctx->d_lfac, lfac.size() * 8), "scratch");
    CK(cudaMemcpy(ctx->d_lfac, lfac.data(), lfac.size() * 8, cudaMemcpyHostToDevice), "upload");
    lu_init_attributes();
    pairs_init_attributes();
    *out = ctx.release();
    return TCU_OK;
}

tcu_status tcu_context_destroy(tcu_context* ctx) {
    if (!ctx) return TCU_OK;
    cudaSetDevice(ctx->device);
    cudaStreamSynchronize(ctx->stream);
    while (!ctx->factors.empty()) tcu_factor_destroy(*ctx->factors.begin());  // factors left alive
    for (tcu_context* w : ctx->workers) tcu_context_destroy(w);
    for (auto& kv : ctx->plans) cudaFree(kv.second->mem);
    ctx->pool.release();
    cudaFree(ctx->d_partial);
    cudaFree(ctx->d_cpartial);
    cudaFree(ctx->d_small);
    cudaFree(ctx->d_csmall);
    cudaFree(ctx->d_status);
    cudaFree(ctx->d_lfac);
    cudaStreamDestroy(ctx->stream);
    delete ctx;
    return TCU_OK;
}

void* tcu_context_stream(tcu_context* ctx) { return ctx ? (void*)ctx->stream : nullptr; }

tcu_status tcu_context_set_profiling(tcu_context* ctx, int enabled) {
    if (!ctx) return fail(TCU_INVALID_INPUT, "null context");
    std::lock_guard<std::recursive_mutex> lock(ctx->mu);
    ctx->prof.on = enabled != 0;
    return TCU_OK;
}
tcu_status tcu_context_stage_time(tcu_context* ctx, int stage, long long* launches, double* total_ms) {
    if (!ctx || stage < 0 || stage >= ST_COUNT || !launches || !total_ms) return fail(TCU_INVALID_INPUT, "bad stage");
    std::lock_guard<std::recursive_mutex> lock(ctx->mu);
    cudaSetDevice(ctx->device);
    ctx->prof.collect();
    *launches = ctx->prof.count[stage];
    *total_ms = ctx->prof.total_ms[stage];
    return TCU_OK;
}
tcu_status tcu_context_reset_stage_times(tcu_context* ctx) {
    if (!ctx) return fail(TCU_INVALID_INPUT, "null context");
    std::lock_guard<std::recursive_mutex> lock(ctx->mu);
    cudaSetDevice(ctx->device);
    ctx->prof.collect();
    for (int i = 0; i < ST_COUNT; ++i) {
        ctx->prof.count[i] = 0;
        ctx->prof.total_ms[i] = 0.0;
    }
    return TCU_OK;
}
long long tcu_context_launches(tcu_context* ctx) { return ctx ? ctx->launches : 0; }
long long tcu_context_fallbacks(tcu_context* ctx) { return ctx ? ctx->fallbacks : 0; }

tcu_status tcu_translation_block(tcu_context* ctx, int lmax, double k, const double* disp, int singular, int helicity,
                                 double* out) {
    if (!ctx || !disp || !out) return fail(TCU_INVALID_INPUT, "null argument");
    if (lmax < 1 || lmax > 10 || !std::isfinite(k) || k <= 0 || !finite_all(disp, 3))
        return fail(TCU_INVALID_INPUT, "require 1 <= lmax <= 10, positive finite k and a finite displacement");
    std::lock_guard<std::recursive_mutex> lock(ctx->mu);
    ProfGuard pg(ctx);
    CK(cudaSetDevice(ctx->device), "device");
    if (singular && disp[0] == 0.0 && disp[1] == 0.0 && disp[2] == 0.0)
        return fail(TCU_INVALID_INPUT, "outgoing spherical waves are singular at zero");
    const DevPlan* P;
    tcu_status s = get_plan(ctx, lmax, &P);
    if (s) return s;
    size_t M = 2 * (size_t)lmax * (lmax + 2);
    DevBuf buf(ctx);
    CK(buf.alloc(M * M * 16), "block");
    launch_block(*P, k, disp, singular != 0, helicity != 0, (cplx*)buf.p, ctx->stream);
    ++ctx->launches;
    CK(cudaMemcpyAsync(out, buf.p, M * M * 16, cudaMemcpyDeviceToHost, ctx->stream), "copy");
    return sync_status(ctx, "translation block");
}

double tcu_wigner3j(int j1, int j2, int j3, int m1, int m2, int m3) {
    if (j1 < 0 || j2 < 0 || j3 < 0 || j1 > 60 || j2 > 60 || j3 > 60) return 0.0;
    return wigner3j_racah(j1, j2, j3, m1, m2, m3);
}

tcu_status tcu_translate(tcu_context* ctx, size_t count, const int* labels, const double* args, int helicity,
                         int singular, double* out) {
    if (!ctx || (count > 0 && (!labels || !args || !out))) return fail(TCU_INVALID_INPUT, "null argument");
    int L = 1;
    for (size_t e = 0; e < count; ++e) {
        const int* lb = labels + 6 * e;
        for (int side = 0; side < 2; ++side) {
            const int l = lb[3 * side], m = lb[3 * side + 1], pol = lb[3 * side + 2];
            if (l < 1 || l > 10 || m < -l || m > l || (pol != 0 && pol != 1))
                return fail(TCU_INVALID_INPUT,
                            "mode labels need 1 <= degree <= 10, |order| <= degree and polarization 0 or 1");
            L = std::max(L, l);
        }
    }
    if (!finite_all(args, 6 * count)) return fail(TCU_INVALID_INPUT, "translation arguments must be finite");
    if (count == 0) return TCU_OK;
    std::lock_guard<std::recursive_mutex> lock(ctx->mu);
    ProfGuard pg(ctx);
    CK(cudaSetDevice(ctx->device), "device");
    const DevPlan* P;
    tcu_status s = get_plan(ctx, L, &P);
    if (s) return s;
    DevBuf buf(ctx);
    Arena ar;
    size_t o_l = ar.add(count * 6 * sizeof(int)), o_a = ar.add(count * 48), o_o = ar.add(count * 16);
    CK(buf.alloc(ar.total), "translation buffers");
    CK(cudaMemcpyAsync(ar.at<void>(buf.p, o_l), labels, count * 6 * sizeof(int), cudaMemcpyHostToDevice, ctx->stream),
       "copy");
    CK(cudaMemcpyAsync(ar.at<void>(buf.p, o_a), args, count * 48, cudaMemcpyHostToDevice, ctx->stream), "copy");
    launch_translate(*P, count, ar.at<int>(buf.p, o_l), ar.at<cplx>(buf.p, o_a), helicity != 0, singular != 0,
                     ar.at<cplx>(buf.p, o_o), ctx->stream);
    ++ctx->launches;
    CK(cudaGetLastError(), "translation coefficients");
    CK(cudaMemcpyAsync(out, ar.at<void>(buf.p, o_o), count * 16, cudaMemcpyDeviceToHost, ctx->stream), "copy");
    return sync_status(ctx, "translation coefficients");
}

tcu_status tcu_mie_blocks(tcu_context* ctx, int lmax, double k0, size_t N, const double* radii, const double* eps,
                          double* out) {
    if (!ctx || !radii || !eps || !out || N == 0) return fail(TCU_INVALID_INPUT, "null argument");
    if (lmax < 1 || lmax > 10 || !std::isfinite(k0) || k0 <= 0)
        return fail(TCU_INVALID_INPUT, "require 1 <= lmax <= 10 and a finite positive k0");
    for (size_t i = 0; i < N; ++i)
        if (!std::isfinite(radii[i]) || radii[i] <= 0) return fail(TCU_INVALID_INPUT, "radii must be finite and positive");
    if (!finite_all(eps, 2 * N)) return fail(TCU_INVALID_INPUT, "permittivities must be finite");
    std::lock_guard<std::recursive_mutex> lock(ctx->mu);
    ProfGuard pg(ctx);
    CK(cudaSetDevice(ctx->device), "device");
    DevBuf buf(ctx);
    Arena ar;
    size_t o_r = ar.add(N * 8), o_e = ar.add(N * 16), o_t = ar.add(N * lmax * 64);
    CK(buf.alloc(ar.total), "mie buffers");
    double* r = ar.at<double>(buf.p, o_r);
    cplx* e = ar.at<cplx>(buf.p, o_e);
    cplx* T = ar.at<cplx>(buf.p, o_t);
    CK(cudaMemcpyAsync(r, radii, N * 8, cudaMemcpyHostToDevice, ctx->stream), "copy");
    CK(cudaMemcpyAsync(e, eps, N * 16, cudaMemcpyHostToDevice, ctx->stream), "copy");
    CK(cudaMemsetAsync(ctx->d_status, 0, 4, ctx->stream), "status");
    launch_mie(lmax, k0, (int)N, r, e, T, ctx->d_status, ctx->stream);
    ++ctx->launches;
    tcu_status s = read_status(ctx, "Mie coefficients");
    if (s) return s;
    CK(cudaMemcpyAsync(out, T, N * lmax * 64, cudaMemcpyDeviceToHost, ctx->stream), "copy");
    return sync_status(ctx, "Mie coefficients");
}

tcu_status tcu_plane_wave_expansion(tcu_context* ctx, int lmax, size_t N, const double* positions, int p,
                                    const double* kvecs, const int* pols, double* out) {
    if (!ctx || !positions || !kvecs || !pols || !out || N == 0 || p <= 0) return fail(TCU_INVALID_INPUT, "null argument");
    if (lmax < 1 || lmax > 10) return fail(TCU_INVALID_INPUT, "require 1 <= lmax <= 10");
    for (int c = 0; c < p; ++c)
        if (pols[c] != 0 && pols[c] != 1) return fail(TCU_INVALID_INPUT, "polarization must be 0 or 1");
    if (!finite_all(kvecs, 6 * p) || !finite_all(positions, 3 * N))
        return fail(TCU_INVALID_INPUT, "wavevector must be finite");
    std::lock_guard<std::recursive_mutex> lock(ctx->mu);
    ProfGuard pg(ctx);
    CK(cudaSetDevice(ctx->device), "device");
    size_t M = 2 * (size_t)lmax * (lmax + 2), n = N * M;
    DevBuf buf(ctx);
    Arena ar;
    size_t o_pos = ar.add(N * 24), o_kv = ar.add(p * 48), o_o = ar.add(n * p * 16), o_pl = ar.add(p * 4);
    CK(buf.alloc(ar.total), "plane-wave buffers");
    double* pos = ar.at<double>(buf.p, o_pos);
    cplx* kv = ar.at<cplx>(buf.p, o_kv);
    cplx* o = ar.at<cplx>(buf.p, o_o);
    int* pl = ar.at<int>(buf.p, o_pl);
    CK(cudaMemcpyAsync(pos, positions, N * 24, cudaMemcpyHostToDevice, ctx->stream), "copy");
    CK(cudaMemcpyAsync(kv, kvecs, p * 48, cudaMemcpyHostToDevice, ctx->stream), "copy");
    CK(cudaMemcpyAsync(pl, pols, p * 4, cudaMemcpyHostToDevice, ctx->stream), "copy");
    launch_plane_wave(lmax, (int)N, pos, p, kv, pl, ctx->d_lfac, o, ctx->stream);
    ++ctx->launches;
    CK(cudaMemcpyAsync(out, o, n * p * 16, cudaMemcpyDeviceToHost, ctx->stream), "copy");
    return sync_status(ctx, "plane-wave expansion");
}

tcu_status tcu_cross_sections(tcu_context* ctx, int lmax, double k0, size_t N, const double* positions, int p,
                              const double* x, const double* b, double* sca, double* ext) {
    if (!ctx || !positions || !x || !b || !sca || !ext || N == 0 || p <= 0) return fail(TCU_INVALID_INPUT, "null argument");
    if (lmax < 1 || lmax > 10 || !std::isfinite(k0) || k0 <= 0) return fail(TCU_INVALID_INPUT, "invalid lmax or k0");
    std::lock_guard<std::recursive_mutex> lock(ctx->mu);
    ProfGuard pg(ctx);
    CK(cudaSetDevice(ctx->device), "device");
    const DevPlan* P;
    tcu_status s = get_plan(ctx, lmax, &P);
    if (s) return s;
    size_t M = 2 * (size_t)lmax * (lmax + 2), n = N * M, per = n * p;
    DevBuf buf(ctx);
    Arena ar;
    size_t o_pos = ar.add(N * 24), o_x = ar.add(3 * per * 16);
    CK(buf.alloc(ar.total), "cross-section buffers");
    double* pos = ar.at<double>(buf.p, o_pos);
    cplx* dx = ar.at<cplx>(buf.p, o_x);
    cplx* db = dx + per;
    cplx* ox = db + per;
    CK(cudaMemcpyAsync(pos, positions, N * 24, cudaMemcpyHostToDevice, ctx->stream), "copy");
    CK(cudaMemcpyAsync(dx, x, per * 16, cudaMemcpyHostToDevice, ctx->stream), "copy");
    CK(cudaMemcpyAsync(db, b, per * 16, cudaMemcpyHostToDevice, ctx->stream), "copy");
    apply_op(ctx, P, (int)N, k0, pos, nullptr, dx, n, p, nullptr, 1.0, 1.0, false, ox);
    std::vector<double> s1(p), s2(p);
    vec_real_dots(dx, ox, n, p, ctx->d_small, ctx->d_partial, ctx->stream);
    CK(cudaMemcpyAsync(s1.data(), ctx->d_small, p * 8, cudaMemcpyDeviceToHost, ctx->stream), "copy");
    vec_real_dots(db, dx, n, p, ctx->d_small + 32, ctx->d_partial + 4 * 256, ctx->stream);
    ctx->launches += 4;
    CK(cudaMemcpyAsync(s2.data(), ctx->d_small + 32, p * 8, cudaMemcpyDeviceToHost, ctx->stream), "copy");
    s = sync_status(ctx, "cross sections");
    if (s) return s;
    for (int c = 0; c < p; ++c) {
        sca[c] = s1[c] / (k0 * k0);
        ext[c] = -s2[c] / (k0 * k0);
    }
    return TCU_OK;
}

tcu_status tcu_sphere_cluster_factor(tcu_context* ctx, int lmax, double k0, size_t N, const double* radii,
                                     const double* eps, const double* positions, int precision, tcu_factor** out) {
    if (!ctx) return fail(TCU_INVALID_INPUT, "null context");
    std::lock_guard<std::recursive_mutex> lock(ctx->mu);
    ProfGuard pg(ctx);
    CK(cudaSetDevice(ctx->device), "device");
    return factor_impl(ctx, lmax, k0, N, radii, eps, positions, nullptr, nullptr, nullptr, precision, out);
}

tcu_status tcu_sphere_cluster_factor_dev(tcu_context* ctx, int lmax, double k0, size_t N, const double* radii,
                                         const double* eps, const double* positions, int precision,
                                         tcu_factor** out) {
    if (!ctx || !radii || !eps || !positions) return fail(TCU_INVALID_INPUT, "null argument");
    std::lock_guard<std::recursive_mutex> lock(ctx->mu);
    ProfGuard pg(ctx);
    CK(cudaSetDevice(ctx->device), "device");
    // validation reads the (small) geometry back to the host
    std::vector<double> r(N), e(2 * N), p(3 * N);
    CK(cudaMemcpyAsync(r.data(), radii, N * 8, cudaMemcpyDeviceToHost, ctx->stream), "copy");
    CK(cudaMemcpyAsync(e.data(), eps, N * 16, cudaMemcpyDeviceToHost, ctx->stream), "copy");
    CK(cudaMemcpyAsync(p.data(), positions, N * 24, cudaMemcpyDeviceToHost, ctx->stream), "copy");
    tcu_status s = sync_status(ctx, "copy");
    if (s) return s;
    return factor_impl(ctx, lmax, k0, N, r.data(), e.data(), p.data(), radii, eps, positions, precision, out);
}

tcu_status tcu_factor_solve(tcu_factor* f, const double* B, int p, double* X, tcu_certificate* certificates) {
    return solve_impl(f, B, p, X, certificates, false);
}
tcu_status tcu_factor_solve_dev(tcu_factor* f, const double* B, int p, double* X, tcu_certificate* certificates) {
    return solve_impl(f, B, p, X, certificates, true);
}
size_t tcu_factor_dimension(const tcu_factor* f) { return f ? f->n : 0; }

tcu_status tcu_factor_interacting_tmatrix(tcu_factor* f, double* X) {
    if (!f || !X) return fail(TCU_INVALID_INPUT, "null argument");
    const size_t n = f->n;
    const int chunk = 256;  // columns per solve (keeps the solve buffers at 6 n chunk complex)
    std::vector<double> eye;
    for (size_t c0 = 0; c0 < n; c0 += chunk) {
        const int w = (int)std::min<size_t>(chunk, n - c0);
        eye.assign(2 * n * w, 0.0);
        for (int c = 0; c < w; ++c) eye[2 * ((size_t)c * n + c0 + c)] = 1.0;
        tcu_status s = solve_impl(f, eye.data(), w, X + 2 * n * c0, nullptr, false);
        if (s) return s;
    }
    return TCU_OK;
}

tcu_status tcu_factor_global_tmatrix(tcu_factor* f, int lmax_global, const double* origin, double* out) {
    if (!f || !origin || !out) return fail(TCU_INVALID_INPUT, "null argument");
    if (lmax_global < 1 || lmax_global > 10 || !finite_all(origin, 3))
        return fail(TCU_INVALID_INPUT, "require 1 <= lmax_global <= 10 and a finite origin");
    tcu_context* ctx = f->ctx;
    std::lock_guard<std::recursive_mutex> lock(ctx->mu);
    ProfGuard pg(ctx);
    CK(cudaSetDevice(ctx->device), "device");
    const int Lmax = std::max(f->L, lmax_global);
    const DevPlan* P;
    tcu_status s = get_plan(ctx, Lmax, &P);
    if (s) return s;
    const size_t n = f->n, Mg = 2 * (size_t)lmax_global * (lmax_global + 2);
    DevBuf buf(ctx);
    Arena ar;
    size_t oO = ar.add(24), oI = ar.add(n * Mg * 16), oY = ar.add(n * Mg * 16), oE = ar.add(n * Mg * 16),
           oT = ar.add(Mg * Mg * 16);
    CK(buf.alloc(ar.total), "expansion buffers");
    double* d_o = ar.at<double>(buf.p, oO);
    cplx* Ein = ar.at<cplx>(buf.p, oI);
    cplx* Y = ar.at<cplx>(buf.p, oY);
    cplx* Eout = ar.at<cplx>(buf.p, oE);
    cplx* Tg = ar.at<cplx>(buf.p, oT);
    CK(cudaMemcpyAsync(d_o, origin, 24, cudaMemcpyHostToDevice, ctx->stream), "copy");
    CK(cudaMemsetAsync(Ein, 0, n * Mg * 16, ctx->stream), "clear");
    CK(cudaMemsetAsync(Eout, 0, n * Mg * 16, ctx->stream), "clear");
    launch_expand_blocks(*P, f->N, f->k0, f->d_pos, origin, f->L * (f->L + 2), lmax_global * (lmax_global + 2), Ein,
                         Eout, ctx->stream);
    ++ctx->launches;
    if ((s = sync_status(ctx, "expansion blocks"))) return s;
    // Y = (I - T C)^-1 T Ein (refined in FP64), T_global = Eout Y
    if ((s = solve_impl(f, (const double*)Ein, (int)Mg, (double*)Y, nullptr, true))) return s;
    launch_zgemm_small((int)Mg, (int)Mg, (int)n, Eout, Mg, Y, n, Tg, Mg, ctx->stream);
    ++ctx->launches;
    CK(cudaMemcpyAsync(out, Tg, Mg * Mg * 16, cudaMemcpyDeviceToHost, ctx->stream), "copy");
    (void)d_o;
    return sync_status(ctx, "global T-matrix");
}

tcu_status tcu_factor_solve_adjoint(tcu_factor* f, const double* G, int p, double* Y, tcu_certificate* certificates) {
    return solve_adjoint_impl(f, G, p, Y, certificates, false);
}
tcu_status tcu_factor_pullback_incident(tcu_factor* f, const double* G, int p, double* out,
                                        tcu_certificate* certificates) {
    return solve_adjoint_impl(f, G, p, out, certificates, true);
}

tcu_status tcu_factor_destroy(tcu_factor* f) {
    if (!f) return TCU_OK;
    if (f->fallback) tcu_factor_destroy(f->fallback);
    cudaSetDevice(f->ctx->device);
    cudaStreamSynchronize(f->ctx->stream);
    {
        std::lock_guard<std::recursive_mutex> lock(f->ctx->mu);
        f->ctx->factors.erase(f);
        for (void* q : {(void*)f->d_pos, (void*)f->d_radii, (void*)f->d_eps, (void*)f->d_T, f->d_A,
                        (void*)f->d_inv, (void*)f->wk.piv, f->wk.pack, (void*)f->d_scale, (void*)f->d_Z})
            f->ctx->pool.free(q);
    }
    delete f;
    return TCU_OK;
}

tcu_status tcu_cluster_operator(tcu_context* ctx, int lmax, double k0, size_t N, const double* radii,
                                const double* eps, const double* positions, double* out) {
    if (!ctx || !out) return fail(TCU_INVALID_INPUT, "null argument");
    std::lock_guard<std::recursive_mutex> lock(ctx->mu);
    ProfGuard pg(ctx);
    CK(cudaSetDevice(ctx->device), "device");
    tcu_status s = validate_spheres(lmax, k0, N, radii, eps, positions);
    if (s) return s;
    const DevPlan* P;
    if ((s = get_plan(ctx, lmax, &P))) return s;
    size_t M = 2 * (size_t)lmax * (lmax + 2), n = N * M;
    DevBuf buf(ctx);
    CK(buf.alloc(N * 24 + N * 8 + N * 16 + N * lmax * 64 + n * n * 16), "operator buffers");
    double* pos = (double*)buf.p;
    double* r = pos + 3 * N;
    cplx* e = (cplx*)(r + N);
    cplx* T = e + N;
    cplx* A = T + N * lmax * 4;
    CK(cudaMemcpyAsync(pos, positions, N * 24, cudaMemcpyHostToDevice, ctx->stream), "copy");
    CK(cudaMemcpyAsync(r, radii, N * 8, cudaMemcpyHostToDevice, ctx->stream), "copy");
    CK(cudaMemcpyAsync(e, eps, N * 16, cudaMemcpyHostToDevice, ctx->stream), "copy");
    CK(cudaMemsetAsync(ctx->d_status, 0, 4, ctx->stream), "status");
    launch_mie(lmax, k0, (int)N, r, e, T, ctx->d_status, ctx->stream);
    if ((s = read_status(ctx, "Mie coefficients"))) return s;
    launch_assemble(*P, (int)N, k0, pos, T, A, n, false, ctx->stream);
    ctx->launches += 2;
    CK(cudaMemcpyAsync(out, A, n * n * 16, cudaMemcpyDeviceToHost, ctx->stream), "copy");
    return sync_status(ctx, "cluster operator");
}

tcu_status tcu_cluster_apply(tcu_context* ctx, int lmax, double k0, size_t N, const double* radii, const double* eps,
                             const double* positions, int p, const double* x, double* y) {
    if (!ctx || !x || !y || p <= 0) return fail(TCU_INVALID_INPUT, "null argument");
    std::lock_guard<std::recursive_mutex> lock(ctx->mu);
    ProfGuard pg(ctx);
    CK(cudaSetDevice(ctx->device), "device");
    tcu_status s = validate_spheres(lmax, k0, N, radii, eps, positions);
    if (s) return s;
    const DevPlan* P;
    if ((s = get_plan(ctx, lmax, &P))) return s;
    size_t M = 2 * (size_t)lmax * (lmax + 2), n = N * M, per = n * p;
    DevBuf buf(ctx);
    CK(buf.alloc(N * 24 + N * 8 + N * 16 + N * lmax * 64 + 2 * per * 16), "apply buffers");
    double* pos = (double*)buf.p;
    double* r = pos + 3 * N;
    cplx* e = (cplx*)(r + N);
    cplx* T = e + N;
    cplx* dx = T + N * lmax * 4;
    cplx* dy = dx + per;
    CK(cudaMemcpyAsync(pos, positions, N * 24, cudaMemcpyHostToDevice, ctx->stream), "copy");
    CK(cudaMemcpyAsync(r, radii, N * 8, cudaMemcpyHostToDevice, ctx->stream), "copy");
    CK(cudaMemcpyAsync(e, eps, N * 16, cudaMemcpyHostToDevice, ctx->stream), "copy");
    CK(cudaMemcpyAsync(dx, x, per * 16, cudaMemcpyHostToDevice, ctx->stream), "copy");
    CK(cudaMemsetAsync(ctx->d_status, 0, 4, ctx->stream), "status");
    launch_mie(lmax, k0, (int)N, r, e, T, ctx->d_status, ctx->stream);
    ++ctx->launches;
    if ((s = read_status(ctx, "Mie coefficients"))) return s;
    // Several columns (or TCU_APPLY=stored): the pair tables once, then the stored-table
    // product per column; one column: the product form (building the tables costs about one
    // application, so storing them gains nothing).
    const char* form = getenv("TCU_APPLY");
    const bool forced = form && strcmp(form, "stored") == 0;
    if (apply_gemm_supported(*P) && (forced || (p >= 2 && use_stored_tables(*P, (int)N)))) {
        DevBuf zbuf(ctx), xfbuf(ctx);
        CK(zbuf.alloc(stored_tables_bytes(*P, (int)N, STORED_FULL)), "stored tables");
        CK(xfbuf.alloc(stored_inputs_bytes(*P, (int)N, STORED_FULL, p)), "packed inputs");
        build_stored_tables(*P, (int)N, k0, pos, STORED_FULL, (cplx*)zbuf.p, ctx->stream);
        launch_apply_stored(*P, (int)N, STORED_FULL, (const cplx*)zbuf.p, T, dx, n, p, nullptr, 1.0, -1.0, dy,
                            (cplx*)xfbuf.p, ctx->d_status, ctx->stream);
        ctx->launches += 3;
    } else {
        apply_op(ctx, P, (int)N, k0, pos, T, dx, n, p, nullptr, 1.0, -1.0, true, dy);
    }
    CK(cudaMemcpyAsync(y, dy, per * 16, cudaMemcpyDeviceToHost, ctx->stream), "copy");
    return read_status(ctx, "cluster apply");
}

}  // extern "C"

// ---- GMRES --------------------------------------------------------------------------------
namespace tcu {

// Restarted GMRES of linalg/gmres.rs:119-347 on device vectors: Arnoldi with two classical
// Gram-Schmidt passes (each a fixed-order batched dot product), Givens rotations and the
// Hessenberg solve on the host, true residual b - A x at every restart. With a right
// preconditioner M the Krylov space is built for A M and x = M y.
// op(in, out): out = A in for one device column (the cluster operator or its adjoint).
tcu_status gmres_device(tcu_context* ctx, const std::function<void(const cplx*, cplx*)>& op, const cplx* rhs, size_t n,
                        const tcu_gmres_options& opt, Preconditioner* pre, cplx* x, cplx* work, tcu_certificate* cert) {
    int restart = (int)std::min<long long>(std::min<long long>(opt.restart, (long long)n), opt.max_iterations);
    cplx* V = work;                       // (restart + 1) * n
    cplx* w = V + (size_t)(restart + 1) * n;
    cplx* r = w + n;
    cplx* z = r + n;                      // preconditioned vector
    cplx* Z = z + n;                      // preconditioned basis (restart * n) when pre
    cudaStream_t st = ctx->stream;
    CK(cudaMemsetAsync(x, 0, n * 16, st), "zero");
    CK(cudaMemcpyAsync(r, rhs, n * 16, cudaMemcpyDeviceToDevice, st), "copy");
    double bnorm = 0, rnorm = 0;
    vec_norms(rhs, n, 1, ctx->d_small, ctx->d_partial, st);
    CK(cudaMemcpyAsync(&bnorm, ctx->d_small, 8, cudaMemcpyDeviceToHost, st), "norm");
    tcu_status s = sync_status(ctx, "gmres");
    if (s) return s;
    rnorm = bnorm;
    double tol = std::max(opt.atol, opt.rtol * bnorm);
    int iterations = 0;
    std::vector<std::complex<double>> h((size_t)(restart + 1) * restart), g(restart + 1);
    std::vector<std::pair<double, std::complex<double>>> rot;
    std::vector<std::complex<double>> hp(restart + 1);
    while (true) {
        cert->iterations = iterations;
        cert->residual_norm = rnorm;
        cert->rhs_norm = bnorm;
        if (std::isfinite(rnorm) && rnorm <= tol) return TCU_OK;
        if (!std::isfinite(rnorm) || iterations >= opt.max_iterations) {
            char msg[256];
            snprintf(msg, sizeof msg, "GMRES did not converge after %d iterations: residual %e, tolerance %e", iterations,
                     rnorm, tol);
            return fail(TCU_NOT_CONVERGED, msg);
        }
        vec_scale_copy(V, r, n, 1.0 / rnorm, st);
        std::fill(h.begin(), h.end(), 0.0);
        std::fill(g.begin(), g.end(), 0.0);
        g[0] = rnorm;
        rot.clear();
        int used = 0;
        for (int j = 0; j < restart; ++j) {
            const cplx* vin = V + (size_t)j * n;
            if (pre) {
                pre->apply(vin, Z + (size_t)j * n, st);
                vin = Z + (size_t)j * n;
            }
            op(vin, w);
            for (int pass = 0; pass < 2; ++pass) {
                vec_dots(V, n, j + 1, w, n, ctx->d_csmall, ctx->d_cpartial, st);
                vec_gemv_sub(w, V, n, j + 1, ctx->d_csmall, n, st);
                CK(cudaMemcpyAsync(hp.data(), ctx->d_csmall, (j + 1) * 16, cudaMemcpyDeviceToHost, st), "dots");
                if ((s = sync_status(ctx, "gmres"))) return s;
                for (int i = 0; i <= j; ++i) h[(size_t)j * (restart + 1) + i] += hp[i];
                ctx->launches += 3;
            }
            double next = 0;
            vec_norms(w, n, 1, ctx->d_small, ctx->d_partial, st);
            CK(cudaMemcpyAsync(&next, ctx->d_small, 8, cudaMemcpyDeviceToHost, st), "norm");
            if ((s = sync_status(ctx, "gmres"))) return s;
            ctx->launches += 2;
            h[(size_t)j * (restart + 1) + j + 1] = next;
            for (size_t i = 0; i < rot.size(); ++i) {
                size_t off = (size_t)j * (restart + 1) + i;
                auto a = h[off], b = h[off + 1];
                h[off] = rot[i].first * a + rot[i].second * b;
                h[off + 1] = -std::conj(rot[i].second) * a + rot[i].first * b;
            }
            size_t dg = (size_t)j * (restart + 1) + j;
            auto a = h[dg], b = h[dg + 1];
            double length = std::hypot(std::abs(a), std::abs(b));
            if (!std::isfinite(length) || length == 0.0)
                return fail(TCU_NOT_CONVERGED, "GMRES Arnoldi breakdown before convergence");
            std::complex<double> phase = std::abs(a) == 0.0 ? 1.0 : a / std::abs(a);
            double c = std::abs(a) / length;
            auto sn = phase * std::conj(b) / length;
            h[dg] = phase * length;
            h[dg + 1] = 0.0;
            rot.push_back({c, sn});
            g[j + 1] = -std::conj(sn) * g[j];
            g[j] *= c;
            used = j + 1;
            iterations += 1;
            if (std::abs(g[j + 1]) <= tol || next == 0.0 || iterations == opt.max_iterations) break;
            vec_scale_copy(V + (size_t)(j + 1) * n, w, n, 1.0 / next, st);
            ++ctx->launches;
        }
        for (int i = used - 1; i >= 0; --i) {
            std::complex<double> tail = 0.0;
            for (int jj = i + 1; jj < used; ++jj) tail += h[(size_t)jj * (restart + 1) + i] * g[jj];
            g[i] = (g[i] - tail) / h[(size_t)i * (restart + 1) + i];
        }
        CK(cudaMemcpyAsync(ctx->d_csmall, g.data(), used * 16, cudaMemcpyHostToDevice, st), "coefficients");
        vec_lincomb(x, pre ? Z : V, n, used, ctx->d_csmall, n, st);
        // true residual r = rhs - A x
        op(x, r);
        vec_sub(r, rhs, r, n, 1, st);
        vec_norms(r, n, 1, ctx->d_small, ctx->d_partial, st);
        CK(cudaMemcpyAsync(&rnorm, ctx->d_small, 8, cudaMemcpyDeviceToHost, st), "norm");
        if ((s = sync_status(ctx, "gmres"))) return s;
        ctx->launches += 4;
    }
}

}  // namespace tcu

extern "C" tcu_status tcu_iterative_solve(tcu_context* ctx, int lmax, double k0, size_t N, const double* radii,
                                          const double* eps, const double* positions, const double* B, int p,
                                          const tcu_gmres_options* options, int preconditioner, double* X,
                                          tcu_certificate* certificates) {
    if (!ctx || !B || !X || p <= 0) return fail(TCU_INVALID_INPUT, "null argument");
    tcu_gmres_options opt = options ? *options : tcu_gmres_options{1e-10, 0.0, 30, 300};
    if (!std::isfinite(opt.rtol) || !std::isfinite(opt.atol) || opt.rtol < 0 || opt.atol < 0 ||
        opt.rtol + opt.atol == 0.0 || opt.restart <= 0 || opt.max_iterations <= 0)
        return fail(TCU_INVALID_INPUT,
                    "GMRES needs finite nonnegative tolerances, a positive tolerance, restart and iteration limit");
    if (preconditioner < 0 || preconditioner > 3) return fail(TCU_INVALID_INPUT, "unknown preconditioner");
    std::lock_guard<std::recursive_mutex> lock(ctx->mu);
    ProfGuard pg(ctx);
    PoolScope ps(&ctx->pool);  // the preconditioner's buffers come from the pool, freed before return
    CK(cudaSetDevice(ctx->device), "device");
    tcu_status s = validate_spheres(lmax, k0, N, radii, eps, positions);
    if (s) return s;
    const DevPlan* P;
    if ((s = get_plan(ctx, lmax, &P))) return s;
    size_t M = 2 * (size_t)lmax * (lmax + 2), n = N * M, per = n * p;
    if (!finite_all(B, 2 * per))
        return fail(TCU_INVALID_INPUT,
                    "incident coefficients must be finite, with one row per local multipole and at least one column");
    int restart = std::min(opt.restart, opt.max_iterations);
    if ((size_t)restart > n) restart = (int)n;
    DevBuf buf(ctx);
    size_t work = (size_t)(2 * restart + 4) * n;
    CK(buf.alloc(N * 24 + N * 8 + N * 16 + N * lmax * 64 + (3 * per + work) * 16), "GMRES buffers");
    double* pos = (double*)buf.p;
    double* r = pos + 3 * N;
    cplx* e = (cplx*)(r + N);
    cplx* T = e + N;
    cplx* b = T + N * lmax * 4;
    cplx* tb = b + per;
    cplx* x = tb + per;
    cplx* wk = x + per;
    CK(cudaMemcpyAsync(pos, positions, N * 24, cudaMemcpyHostToDevice, ctx->stream), "copy");
    CK(cudaMemcpyAsync(r, radii, N * 8, cudaMemcpyHostToDevice, ctx->stream), "copy");
    CK(cudaMemcpyAsync(e, eps, N * 16, cudaMemcpyHostToDevice, ctx->stream), "copy");
    CK(cudaMemcpyAsync(b, B, per * 16, cudaMemcpyHostToDevice, ctx->stream), "copy");
    CK(cudaMemsetAsync(ctx->d_status, 0, 4, ctx->stream), "status");
    launch_mie(lmax, k0, (int)N, r, e, T, ctx->d_status, ctx->stream);
    ++ctx->launches;
    if ((s = read_status(ctx, "Mie coefficients"))) return s;
    launch_apply_t(lmax, (int)N, T, b, p, tb, ctx->stream);
    ++ctx->launches;
    // the harmonic tables of all pairs, built once for the applications of every column; launched
    // first, so that the device builds them while the host sets up the preconditioner's graph
    DevBuf zbuf(ctx), xfbuf(ctx);
    const cplx* Zst = nullptr;
    if (use_stored_tables(*P, (int)N)) {
        if (zbuf.alloc(stored_tables_bytes(*P, (int)N, STORED_FULL)) == cudaSuccess &&
            xfbuf.alloc(stored_inputs_bytes(*P, (int)N, STORED_FULL, 1)) == cudaSuccess) {
            build_stored_tables(*P, (int)N, k0, pos, STORED_FULL, (cplx*)zbuf.p, ctx->stream);
            ++ctx->launches;
            Zst = (const cplx*)zbuf.p;
        } else {
            cudaGetLastError();  // no room: the on-the-fly product
        }
    }
    std::unique_ptr<Preconditioner> pre;
    if (preconditioner == TCU_PRECOND_BLOCK_JACOBI) {
        s = make_block_jacobi(ctx->stream, *P, (int)N, k0, pos, positions, radii, T, &pre, &ctx->launches);
        if (s == TCU_OUT_OF_MEMORY) return fail(s, "preconditioner: out of device memory");
        if (s == TCU_SINGULAR) return fail(s, "preconditioner: a diagonal block is numerically singular");
        if (s) return fail(s, "preconditioner set-up failed");
    } else if (preconditioner == TCU_PRECOND_LEARNED || preconditioner == TCU_PRECOND_TWO_LEVEL) {
        std::unique_ptr<CoarseSolve> coarse;
        if ((s = make_coarse(ctx, k0, N, radii, eps, positions, &coarse)))
            return fail(s, std::string("coarse dipole system: ") + g_last_error);
        s = make_two_level(ctx->stream, preconditioner == TCU_PRECOND_LEARNED, *P, lmax, (int)N, k0, pos, positions,
                           radii, eps, T, ctx->precond_reach, ctx->learned_weights, std::move(coarse), &pre,
                           &ctx->launches);
        if (s == TCU_OUT_OF_MEMORY) return fail(s, "two-level preconditioner: out of device memory");
        if (s) return fail(s, "two-level preconditioner set-up failed");
    }
    tcu_status worst = TCU_OK;
    std::string msg;
    for (int c = 0; c < p; ++c) {
        tcu_certificate cert{};
        auto op = [&](const cplx* in, cplx* out) {
            if (Zst) {
                launch_apply_stored(*P, (int)N, STORED_FULL, Zst, T, in, n, 1, nullptr, 1.0, -1.0, out, (cplx*)xfbuf.p,
                                    ctx->d_status, ctx->stream);
                ctx->launches += 2;
            } else {
                launch_apply(*P, (int)N, k0, pos, T, in, n, 1, nullptr, 1.0, -1.0, true, out, ctx->stream);
                ++ctx->launches;
            }
        };
        s = gmres_device(ctx, op, tb + c * n, n, opt, pre.get(), x + c * n, wk, &cert);
        if (certificates) certificates[c] = cert;
        if (s && !worst) {
            worst = s;
            msg = g_last_error;
        }
    }
    CK(cudaMemcpyAsync(X, x, per * 16, cudaMemcpyDeviceToHost, ctx->stream), "copy");
    s = read_status(ctx, "GMRES");
    if (s) return s;
    if (worst) return fail(worst, msg);
    return TCU_OK;
}

extern "C" tcu_status tcu_iterative_pullback_incident(tcu_context* ctx, int lmax, double k0, size_t N,
                                                      const double* radii, const double* eps, const double* positions,
                                                      const double* G, int p, const tcu_gmres_options* options,
                                                      double* out, tcu_certificate* certificates) {
    if (!ctx || !G || !out || p <= 0) return fail(TCU_INVALID_INPUT, "null argument");
    tcu_gmres_options opt = options ? *options : tcu_gmres_options{1e-10, 0.0, 30, 300};
    if (!std::isfinite(opt.rtol) || !std::isfinite(opt.atol) || opt.rtol < 0 || opt.atol < 0 ||
        opt.rtol + opt.atol == 0.0 || opt.restart <= 0 || opt.max_iterations <= 0)
        return fail(TCU_INVALID_INPUT,
                    "GMRES needs finite nonnegative tolerances, a positive tolerance, restart and iteration limit");
    std::lock_guard<std::recursive_mutex> lock(ctx->mu);
    ProfGuard pg(ctx);
    CK(cudaSetDevice(ctx->device), "device");
    tcu_status s = validate_spheres(lmax, k0, N, radii, eps, positions);
    if (s) return s;
    const DevPlan* P;
    if ((s = get_plan(ctx, lmax, &P))) return s;
    const size_t M = 2 * (size_t)lmax * (lmax + 2), n = N * M, per = n * p;
    if (!finite_all(G, 2 * per)) return fail(TCU_INVALID_INPUT, "invalid illumination cotangent");
    int restart = std::min(opt.restart, opt.max_iterations);
    if ((size_t)restart > n) restart = (int)n;
    DevBuf buf(ctx);
    const size_t work = (size_t)(2 * restart + 4) * n;
    Arena ar;
    size_t oP = ar.add(N * 24), oR = ar.add(N * 8), oE = ar.add(N * 16), oT = ar.add(N * lmax * 64),
           oG = ar.add(per * 16), oY = ar.add(per * 16), oW = ar.add(work * 16), o1 = ar.add(n * 16), o2 = ar.add(n * 16);
    CK(buf.alloc(ar.total), "adjoint GMRES buffers");
    double* pos = ar.at<double>(buf.p, oP);
    double* r = ar.at<double>(buf.p, oR);
    cplx* e = ar.at<cplx>(buf.p, oE);
    cplx* T = ar.at<cplx>(buf.p, oT);
    cplx* g = ar.at<cplx>(buf.p, oG);
    cplx* y = ar.at<cplx>(buf.p, oY);
    cplx* wk = ar.at<cplx>(buf.p, oW);
    cplx* t1 = ar.at<cplx>(buf.p, o1);
    cplx* t2 = ar.at<cplx>(buf.p, o2);
    CK(cudaMemcpyAsync(pos, positions, N * 24, cudaMemcpyHostToDevice, ctx->stream), "copy");
    CK(cudaMemcpyAsync(r, radii, N * 8, cudaMemcpyHostToDevice, ctx->stream), "copy");
    CK(cudaMemcpyAsync(e, eps, N * 16, cudaMemcpyHostToDevice, ctx->stream), "copy");
    CK(cudaMemcpyAsync(g, G, per * 16, cudaMemcpyHostToDevice, ctx->stream), "copy");
    CK(cudaMemsetAsync(ctx->d_status, 0, 4, ctx->stream), "status");
    launch_mie(lmax, k0, (int)N, r, e, T, ctx->d_status, ctx->stream);
    ++ctx->launches;
    if ((s = read_status(ctx, "Mie coefficients"))) return s;
    // the pair tables, stored once for every application of the adjoint operator
    DevBuf zbuf(ctx), xfbuf(ctx);
    const cplx* Zst = nullptr;
    if (use_stored_tables(*P, (int)N)) {
        if (zbuf.alloc(stored_tables_bytes(*P, (int)N, STORED_FULL)) == cudaSuccess &&
            xfbuf.alloc(stored_inputs_bytes(*P, (int)N, STORED_FULL, 1)) == cudaSuccess) {
            build_stored_tables(*P, (int)N, k0, pos, STORED_FULL, (cplx*)zbuf.p, ctx->stream);
            ++ctx->launches;
            Zst = (const cplx*)zbuf.p;
        } else {
            cudaGetLastError();  // no room: the on-the-fly product
        }
    }
    auto op = [&](const cplx* in, cplx* o) {
        launch_apply_adjoint(*P, (int)N, k0, pos, T, in, n, 1, o, t1, t2, ctx->stream, &ctx->launches, Zst,
                             (cplx*)xfbuf.p, ctx->d_status);
    };
    tcu_status worst = TCU_OK;
    std::string msg;
    for (int c = 0; c < p; ++c) {
        tcu_certificate cert{};
        s = gmres_device(ctx, op, g + c * n, n, opt, nullptr, y + c * n, wk, &cert);
        if (certificates) certificates[c] = cert;
        if (s && !worst) {
            worst = s;
            msg = g_last_error;
        }
    }
    launch_apply_th(lmax, (int)N, T, y, n, p, g, ctx->stream);  // the incident gradient T^H Y
    ++ctx->launches;
    CK(cudaMemcpyAsync(out, g, per * 16, cudaMemcpyDeviceToHost, ctx->stream), "copy");
    s = read_status(ctx, "adjoint GMRES");
    if (s) return s;
    if (worst) return fail(worst, msg);
    return TCU_OK;
}

// =========================================================================================
// 2D lattice sums at shift 0 and the batched periodic-array solve.
namespace {

double log_fact(int n) { return std::lgamma((double)n + 1.0); }

// Host-side set-up of one batch of lattice sums: split, lattice points within the real-space
// cutoff, reciprocal vectors within the reciprocal cutoff, and the per-(l, m) constants.
// Double-double arithmetic (Dekker's two-product via fma, Knuth's two-sum; Bailey's division) for
// the reciprocal lattice vectors: next to a diffraction threshold q.q - k^2 resolves digits that a
// binary64 reciprocal vector b = 2 pi a / det rounds away.
struct DD {
    double hi, lo;
};
DD dd_two_sum(double a, double b) {
    const double s = a + b, z = s - a;
    return {s, (a - (s - z)) + (b - z)};
}
DD dd_norm(double hi, double lo) {
    const double s = hi + lo;
    return {s, lo - (s - hi)};
}
DD dd_add(DD a, DD b) {
    const DD s = dd_two_sum(a.hi, b.hi);
    return dd_norm(s.hi, s.lo + a.lo + b.lo);
}
DD dd_mul(DD a, double b) {
    const double p = a.hi * b;
    return dd_norm(p, std::fma(a.hi, b, -p) + a.lo * b);
}
DD dd_div(DD a, DD b) {
    const double q1 = a.hi / b.hi;
    const DD r = dd_add(a, dd_mul(b, -q1));
    const double q2 = r.hi / b.hi;
    const DD r2 = dd_add(r, dd_mul(b, -q2));
    return dd_add(dd_two_sum(q1, q2), DD{r2.hi / b.hi, 0.0});
}
// reciprocal vectors b1 = 2 pi (a2y, -a2x)/det, b2 = 2 pi (-a1y, a1x)/det of the binary64 lattice
void reciprocal_dd(const double* lat, DD b[2][2]) {
    const DD twopi{6.283185307179586, 2.4492935982947064e-16};
    const DD p = dd_two_sum(lat[0] * lat[3], 0.0), q = dd_two_sum(lat[1] * lat[2], 0.0);
    const DD det = dd_add(dd_add(p, DD{std::fma(lat[0], lat[3], -p.hi), 0.0}),
                          dd_mul(dd_add(q, DD{std::fma(lat[1], lat[2], -q.hi), 0.0}), -1.0));
    b[0][0] = dd_div(dd_mul(twopi, lat[3]), det);
    b[0][1] = dd_div(dd_mul(twopi, -lat[2]), det);
    b[1][0] = dd_div(dd_mul(twopi, -lat[1]), det);
    b[1][1] = dd_div(dd_mul(twopi, lat[0]), det);
}

struct LatticeSetup {
    double eta = 0, area = 0;
    double sx = 0, sy = 0;      // in-plane shift reduced into the cell, r' = r - R0
    double sz = 0;              // shift off the lattice plane
    double R0x = 0, R0y = 0;    // the lattice vector taken off (Bloch phase e^{-i kpar.R0})
    bool at_origin = true;      // r' = 0: the self term, and no R = 0 real-space term
    double t = 0;               // (k r_z eta)^2 of the t-series off the plane
    int J = 0;                  // its last term
    std::vector<double2> R, G, Glo;  // Glo: low parts of the reciprocal vectors
    std::vector<double> norm, reflection, coef, coefz;
    std::vector<double2> pref;
    double2 self0{0, 0};
};

tcu_status lattice_setup(int lsum, double k, const double* lat, size_t nk, const double* kpars, double eta_in,
                         LatticeSetup& S, const double* shift = nullptr) {
    if (lsum < 0 || lsum > LS_MAXL) return fail(TCU_INVALID_INPUT, "require 0 <= lmax_sum <= 14");
    if (!std::isfinite(k) || k <= 0.0)
        return fail(TCU_INVALID_INPUT, "the device lattice sums take a positive real wavenumber");
    if (!lat || !finite_all(lat, 4) || nk == 0 || !kpars || !finite_all(kpars, 2 * nk))
        return fail(TCU_INVALID_INPUT, "lattice must be a finite 2 x 2 matrix with finite Bloch vectors");
    const double a1x = lat[0], a1y = lat[1], a2x = lat[2], a2y = lat[3];
    const double det = a1x * a2y - a1y * a2x;
    S.area = std::fabs(det);
    if (!(S.area > 0.0) || !std::isfinite(S.area)) return fail(TCU_INVALID_INPUT, "lattice is numerically singular");
    double eta = eta_in;
    if (!std::isfinite(eta) || eta < 0.0) return fail(TCU_INVALID_INPUT, "the device lattice sums take a real split >= 0");
    if (eta == 0.0) {  // lattice/cell.rs:164-175
        double kl = k * std::sqrt(S.area);
        eta = std::sqrt(2.0 * M_PI) / kl * std::max(kl / 8.0, 1.0);
    }
    // Off the plane the t-series cancels to about e^(-|t|/2) of its largest term, so the split is
    // capped at |t| = (k r_z eta)^2 <= 1 where 1/(2 eta^2) <= 8 allows (the sum does not depend on it)
    if (shift && shift[2] != 0.0) eta = std::min(eta, std::max(0.25, 1.0 / std::fabs(k * shift[2])));
    const double c = 0.5 / (eta * eta);
    if (c > 8.0)
        return fail(TCU_INVALID_INPUT,
                    "Ewald split too small for the device lattice sums (require 1/(2 eta^2) <= 8); eta = 0 selects one");
    S.eta = eta;
    if (shift) {
        // reduce the shift into the cell (lattice/ewald.rs:610-665): r' = r - R0 with R0 the lattice
        // vector of the rounded fractional coordinates, and the phase e^{-i kpar.R0} on the result
        const double f0 = (a2y * shift[0] - a2x * shift[1]) / det, f1 = (-a1y * shift[0] + a1x * shift[1]) / det;
        const double c0 = std::round(f0), c1 = std::round(f1);
        S.R0x = c0 * a1x + c1 * a2x;
        S.R0y = c0 * a1y + c1 * a2y;
        S.sx = shift[0] - S.R0x;
        S.sy = shift[1] - S.R0y;
        S.sz = shift[2];
        S.at_origin = S.sx == 0.0 && S.sy == 0.0 && S.sz == 0.0;
    }
    // off the plane: F_(1/2-n)(v, t) = sum_j (t/2)^j / j! F_(1/2-n-j)(v, 0) (lattice/reduced.rs:223),
    // terms until (t/2)^j / j! falls below 1e-18 of the largest; the alternating limits cancel
    // to about e^(-t/2) of the largest term, so t is bounded to keep FP64 accuracy
    double zabs = 0.0;
    if (S.sz != 0.0) {
        zabs = std::fabs(k * S.sz);
        S.t = (zabs * eta) * (zabs * eta);
        if (!(S.t <= 16.0))
            return fail(TCU_INVALID_INPUT,
                        "shift too far off the lattice plane for the device lattice sums (require (k r_z eta)^2 <= 16)");
        double term = 1.0, big = 1.0;
        int J = 1;
        for (; J < LS_TMAX; ++J) {
            term *= 0.5 * S.t / J;
            big = std::max(big, term);
            if (J > 0.5 * S.t && term < 1e-18 * big) break;
        }
        S.J = J;
    }
    const double ke = k * eta;
    // real space: Gaussian factor e^{-(k eta)^2 R^2/2 + c} below e^-46 times the polynomial growth
    double Rc = std::sqrt(2.0 * (46.0 + c) / (ke * ke));
    for (int it = 0; it < 30; ++it)
        Rc = std::sqrt(2.0 * (46.0 + c + lsum * std::log(std::max(1.0, k * Rc)) +
                              (2 * lsum + 1) * std::log(std::max(1.0, eta))) /
                       (ke * ke));
    const double len1 = std::hypot(a1x, a1y), len2 = std::hypot(a2x, a2y);
    const double hdir = S.area / std::max(len1, len2);
    const double rin = std::hypot(S.sx, S.sy);
    long Nd = (long)std::ceil((Rc + rin) / hdir) + 1;
    if (Nd > 64) return fail(TCU_INVALID_INPUT, "lattice too elongated for the device lattice sums");
    for (long s = S.at_origin ? 1 : 0; s <= Nd; ++s)  // cube shells, fixed order; R = 0 when shifted
        for (long n1 = -s; n1 <= s; ++n1)
            for (long n2 = -s; n2 <= s; ++n2) {
                if (std::max(std::labs(n1), std::labs(n2)) != s) continue;
                double x = n1 * a1x + n2 * a2x, y = n1 * a1y + n2 * a2y;
                if (std::hypot(x + S.sx, y + S.sy) <= Rc) S.R.push_back(make_double2(x, y));
            }
    // reciprocal: e^{-v} (q/k)^lsum (2 eta^2)^n below e^-46 (off the plane also times the
    // growth e^(t/2) of the t-series terms and the powers of k r_z)
    const double b1x = 2 * M_PI * a2y / det, b1y = -2 * M_PI * a2x / det;
    const double b2x = -2 * M_PI * a1y / det, b2y = 2 * M_PI * a1x / det;
    const double budget = 46.0 + 0.5 * S.t + lsum * std::log(std::max(1.0, zabs));
    double x2 = 1.0 + 2.0 * eta * eta * budget;
    for (int it = 0; it < 30; ++it)
        x2 = 1.0 + 2.0 * eta * eta *
                       (budget + 0.5 * lsum * std::log(std::max(1.0, x2)) +
                        (lsum / 2) * std::log(std::max(1.0, 2.0 * eta * eta)) + std::log(std::max(1.0, 1.0 / eta)));
    double kmax = 0.0;
    for (size_t i = 0; i < nk; ++i) kmax = std::max(kmax, std::hypot(kpars[2 * i], kpars[2 * i + 1]));
    const double qc = k * std::sqrt(x2) + kmax;
    const double blen1 = std::hypot(b1x, b1y), blen2 = std::hypot(b2x, b2y);
    const double hrec = (4 * M_PI * M_PI / S.area) / std::max(blen1, blen2);
    long Nr = (long)std::ceil(qc / hrec) + 1;
    if (Nr > 64) return fail(TCU_INVALID_INPUT, "lattice or Bloch vectors out of range for the device lattice sums");
    DD bdd[2][2];
    reciprocal_dd(lat, bdd);
    for (long s = 0; s <= Nr; ++s)
        for (long n1 = -s; n1 <= s; ++n1)
            for (long n2 = -s; n2 <= s; ++n2) {
                if (std::max(std::labs(n1), std::labs(n2)) != s) continue;
                const DD x = dd_add(dd_mul(bdd[0][0], (double)n1), dd_mul(bdd[1][0], (double)n2));
                const DD y = dd_add(dd_mul(bdd[0][1], (double)n1), dd_mul(bdd[1][1], (double)n2));
                if (std::hypot(x.hi, y.hi) <= qc) {
                    S.G.push_back(make_double2(x.hi, y.hi));
                    S.Glo.push_back(make_double2(x.lo, y.lo));
                }
            }
    const int T = (lsum + 1) * (lsum + 1);
    S.norm.assign(T, 0.0);
    S.reflection.assign(T, 0.0);
    S.coef.assign((size_t)T * LS_NMAX, 0.0);
    S.pref.assign(T, make_double2(0, 0));
    for (int l = 0; l <= lsum; ++l)
        for (int m = -l; m <= l; ++m) {
            int lm = l * l + l + m, am = std::abs(m);
            S.norm[lm] = std::sqrt((2 * l + 1) / (4 * M_PI)) * std::exp(0.5 * (log_fact(l - m) - log_fact(l + m)));
            S.reflection[lm] = ((am % 2) ? -1.0 : 1.0) * std::exp(log_fact(l - am) - log_fact(l + am));
            if ((l - am) % 2 == 0)
                for (int n = 0; n <= (l - am) / 2; ++n)
                    S.coef[(size_t)lm * LS_NMAX + n] =
                        std::exp(-log_fact(n) - log_fact((l + am - 2 * n) / 2) - log_fact((l - am - 2 * n) / 2));
            if (S.sz != 0.0) {
                // S_lmn off the plane (reciprocal.rs:22-60): coefficient of beta^(2p), p = (l-|m|-s)/2,
                // (-k r_z)^(2n-s) / ((2n-s)! (s-n)! ((l+|m|-s)/2)! ((l-|m|-s)/2)!), n <= s <= min(l-|m|, 2n)
                if (S.coefz.empty()) S.coefz.assign((size_t)T * LS_PMAX * LS_FMAX, 0.0);
                const double mz = -k * S.sz;
                for (int n = 0; n <= l - am; ++n)
                    for (int sidx = n; sidx <= std::min(l - am, 2 * n); ++sidx) {
                        if ((l - am - sidx) % 2) continue;
                        const int p = (l - am - sidx) / 2;
                        S.coefz[((size_t)lm * LS_PMAX + p) * LS_FMAX + n] =
                            std::pow(mz, 2 * n - sidx) * std::exp(-log_fact(2 * n - sidx) - log_fact(sidx - n) -
                                                                  log_fact(p + am) - log_fact(p));
                    }
            }
            // sqrt(2l+1) (-i)^m sqrt((l+m)!(l-m)!) / (A k^2 (-2)^l)   (reciprocal.rs:320-330)
            double mag = std::sqrt(2.0 * l + 1.0) * std::exp(0.5 * (log_fact(l + m) + log_fact(l - m))) /
                         (S.area * k * k * std::pow(-2.0, l));
            int ph = ((m % 4) + 4) % 4;  // (-i)^m
            double re = ph == 0 ? 1 : ph == 2 ? -1 : 0, im = ph == 1 ? -1 : ph == 3 ? 1 : 0;
            S.pref[lm] = make_double2(mag * re, mag * im);
        }
    // self term (reciprocal.rs:467-487) at l = 0: Y_00 / (2 sqrt pi) Gamma(-1/2, -1/(2 eta^2) - 0i);
    // Gamma(-1/2, -y - 0i) = Gamma(-1/2) - i y^(-1/2) sum_k y^k / (k! (k - 1/2))
    {
        double y = c, s = 0.0, term = 1.0;
        for (int kk = 0; kk < 400; ++kk) {
            if (kk > 0) term *= y / kk;
            double add = term / (kk - 0.5);
            s += add;
            if (kk > y && std::fabs(add) < 1e-18 * std::fabs(s)) break;
        }
        double gre = -2.0 * std::sqrt(M_PI), gim = -s / std::sqrt(y);
        double f = S.norm[0] * 0.5 / std::sqrt(M_PI);
        S.self0 = make_double2(f * gre, f * gim);
    }
    return TCU_OK;
}

// D (device, nk x T) for device Bloch vectors; shares one LatticeSetup
tcu_status lattice_sums_device(tcu_context* ctx, int lsum, double k, const LatticeSetup& S, size_t nk,
                               const double2* d_kpar, double2* d_out, Arena* scratch_arena, DevBuf& scratch) {
    (void)scratch_arena;
    const int T = (lsum + 1) * (lsum + 1);
    const bool offplane = !S.coefz.empty();
    if (lattice_sum_smem(lsum, (int)S.R.size(), offplane) > 200 * 1024 || S.G.size() > (1u << 20))
        return fail(TCU_INVALID_INPUT, "lattice too elongated for the device lattice sums");
    Arena ar;
    size_t oR = ar.add(S.R.size() * 16), oG = ar.add(S.G.size() * 16), oN = ar.add(T * 8), oRf = ar.add(T * 8),
           oC = ar.add((size_t)T * LS_NMAX * 8), oP = ar.add(T * 16), oTab = ar.add(S.R.size() * T * 16),
           oZ = ar.add(S.coefz.size() * 8), oGl = ar.add(S.Glo.size() * 16);
    CK(scratch.alloc(ar.total), "lattice scratch");
    void* b = scratch.p;
    CK(cudaMemcpyAsync(ar.at<void>(b, oR), S.R.data(), S.R.size() * 16, cudaMemcpyHostToDevice, ctx->stream), "copy");
    CK(cudaMemcpyAsync(ar.at<void>(b, oG), S.G.data(), S.G.size() * 16, cudaMemcpyHostToDevice, ctx->stream), "copy");
    CK(cudaMemcpyAsync(ar.at<void>(b, oGl), S.Glo.data(), S.Glo.size() * 16, cudaMemcpyHostToDevice, ctx->stream),
       "copy");
    CK(cudaMemcpyAsync(ar.at<void>(b, oN), S.norm.data(), T * 8, cudaMemcpyHostToDevice, ctx->stream), "copy");
    CK(cudaMemcpyAsync(ar.at<void>(b, oRf), S.reflection.data(), T * 8, cudaMemcpyHostToDevice, ctx->stream), "copy");
    CK(cudaMemcpyAsync(ar.at<void>(b, oC), S.coef.data(), (size_t)T * LS_NMAX * 8, cudaMemcpyHostToDevice, ctx->stream),
       "copy");
    CK(cudaMemcpyAsync(ar.at<void>(b, oP), S.pref.data(), T * 16, cudaMemcpyHostToDevice, ctx->stream), "copy");
    if (offplane)
        CK(cudaMemcpyAsync(ar.at<void>(b, oZ), S.coefz.data(), S.coefz.size() * 8, cudaMemcpyHostToDevice,
                           ctx->stream),
           "copy");
    CK(cudaMemsetAsync(ctx->d_status, 0, 4, ctx->stream), "status");
    double2* tab = ar.at<double2>(b, oTab);
    launch_real_table(lsum, k, S.eta, (int)S.R.size(), ar.at<double2>(b, oR), S.sx, S.sy, S.sz, ar.at<double>(b, oN),
                      ar.at<double>(b, oRf), tab, ctx->stream);
    ++ctx->launches;
    LatticeSumArgs a;
    a.lsum = lsum;
    a.k = k;
    a.eta = S.eta;
    a.NR = (int)S.R.size();
    a.R = ar.at<double2>(b, oR);
    a.realtab = tab;
    a.NG = (int)S.G.size();
    a.G = ar.at<double2>(b, oG);
    a.Glo = ar.at<double2>(b, oGl);
    a.coef = ar.at<double>(b, oC);
    a.pref = ar.at<double2>(b, oP);
    a.self0 = S.at_origin ? S.self0 : make_double2(0.0, 0.0);
    a.sx = S.sx;
    a.sy = S.sy;
    a.R0x = S.R0x;
    a.R0y = S.R0y;
    a.offplane = offplane ? 1 : 0;
    a.J = S.J;
    a.t = S.t;
    a.coefz = offplane ? ar.at<double>(b, oZ) : nullptr;
    a.nk = (int)nk;
    a.kpar = d_kpar;
    a.out = d_out;
    a.ldo = T;
    a.status = ctx->d_status;
    int grid = (int)std::min<size_t>(nk, 148 * 8);
    launch_lattice_sum(a, grid, ctx->stream);
    ++ctx->launches;
    int st = 0;
    CK(cudaMemcpyAsync(&st, ctx->d_status, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream), "status");
    tcu_status s = sync_status(ctx, "lattice sums");
    if (s) return s;
    if (st == 9)
        return fail(TCU_INVALID_INPUT, "lattice sum is at a diffraction threshold; supply a limiting complex wavenumber");
    if (st) return fail(TCU_DEVICE_ERROR, "lattice sums: device status " + std::to_string(st));
    return TCU_OK;
}

tcu_status array_solve_device(tcu_context* ctx, int lmax, double k0, double radius, const double* eps,
                              const double* lattice, size_t nk, const double2* d_kpar, double eta,
                              const double* kpars_host, double2* d_X) {
    if (lmax < 1 || lmax > 6) return fail(TCU_INVALID_INPUT, "the batched array solve takes 1 <= lmax <= 6");
    if (!std::isfinite(radius) || radius <= 0.0 || !eps || !finite_all(eps, 2))
        return fail(TCU_INVALID_INPUT, "require a positive finite radius and a finite permittivity");
    LatticeSetup S;
    tcu_status s = lattice_setup(2 * lmax, k0, lattice, nk, kpars_host, eta, S);
    if (s) return s;
    double rmin = 1e300;
    for (auto& R : S.R) rmin = std::min(rmin, std::hypot(R.x, R.y));
    if (!(2.0 * radius < rmin))
        return fail(TCU_INVALID_INPUT, "spherical particles must not touch or overlap their lattice images");
    const DevPlan* P = nullptr;
    if ((s = get_plan(ctx, lmax, &P))) return s;
    const int T = (2 * lmax + 1) * (2 * lmax + 1);
    Arena ar;
    size_t oD = ar.add(nk * T * 16), oT = ar.add(lmax * 4 * 16), oE = ar.add(16), oRad = ar.add(8), oN = ar.add(T * 8);
    DevBuf work(ctx), scratch(ctx);
    CK(work.alloc(ar.total), "array-solve workspace");
    void* b = work.p;
    double2* D = ar.at<double2>(b, oD);
    CK(cudaMemcpyAsync(ar.at<void>(b, oE), eps, 16, cudaMemcpyHostToDevice, ctx->stream), "copy");
    CK(cudaMemcpyAsync(ar.at<void>(b, oRad), &radius, 8, cudaMemcpyHostToDevice, ctx->stream), "copy");
    CK(cudaMemcpyAsync(ar.at<void>(b, oN), S.norm.data(), T * 8, cudaMemcpyHostToDevice, ctx->stream), "copy");
    if ((s = lattice_sums_device(ctx, 2 * lmax, k0, S, nk, d_kpar, D, nullptr, scratch))) return s;
    CK(cudaMemsetAsync(ctx->d_status, 0, 4, ctx->stream), "status");
    double2* Tm = ar.at<double2>(b, oT);
    launch_mie(lmax, k0, 1, ar.at<double>(b, oRad), ar.at<cplx>(b, oE), Tm, ctx->d_status, ctx->stream);
    ++ctx->launches;
    if ((s = read_status(ctx, "Mie coefficients"))) return s;
    int grid = (int)std::min<size_t>(nk, 148 * 4);
    launch_array_solve(*P, D, T, ar.at<double>(b, oN), Tm, (int)nk, d_X, ctx->d_status, grid, ctx->stream);
    ++ctx->launches;
    return read_status(ctx, "periodic array solve");
}

}  // namespace

extern "C" tcu_status tcu_lsumsw2d_shift_batch(tcu_context* ctx, int lmax_sum, double k, const double* lattice,
                                               size_t nk, const double* kpars, const double* shift, double eta,
                                               double* out) {
    if (!ctx || !out || !shift) return fail(TCU_INVALID_INPUT, "null context, shift or output");
    if (!finite_all(shift, 3)) return fail(TCU_INVALID_INPUT, "the shift must be finite");
    std::lock_guard<std::recursive_mutex> lock(ctx->mu);
    cudaSetDevice(ctx->device);
    ProfGuard pg(ctx);
    LatticeSetup S;
    tcu_status s = lattice_setup(lmax_sum, k, lattice, nk, kpars, eta, S, shift);
    if (s) return s;
    const int T = (lmax_sum + 1) * (lmax_sum + 1);
    Arena ar;
    size_t oK = ar.add(nk * 16), oO = ar.add(nk * T * 16);
    DevBuf io(ctx), scratch(ctx);
    CK(io.alloc(ar.total), "lattice-sum buffers");
    CK(cudaMemcpyAsync(ar.at<void>(io.p, oK), kpars, nk * 16, cudaMemcpyHostToDevice, ctx->stream), "copy");
    if ((s = lattice_sums_device(ctx, lmax_sum, k, S, nk, ar.at<double2>(io.p, oK), ar.at<double2>(io.p, oO), nullptr,
                                 scratch)))
        return s;
    CK(cudaMemcpyAsync(out, ar.at<void>(io.p, oO), nk * T * 16, cudaMemcpyDeviceToHost, ctx->stream), "copy");
    return sync_status(ctx, "lattice sums");
}

extern "C" tcu_status tcu_lsumsw2d_batch(tcu_context* ctx, int lmax_sum, double k, const double* lattice, size_t nk,
                                         const double* kpars, double eta, double* out) {
    const double zero[3] = {0.0, 0.0, 0.0};
    return tcu_lsumsw2d_shift_batch(ctx, lmax_sum, k, lattice, nk, kpars, zero, eta, out);
}

namespace {

// Host set-up of the complex-wavenumber sums: the split, the shift reduced into the cell, the
// lattice points of both parts within their cutoffs, the S_lmn coefficients with the powers of
// -k r_z folded in, the prefactors and the self term.
struct LatticeSetupCk {
    double eta = 0, area = 0;
    double sx = 0, sy = 0, sz = 0, R0x = 0, R0y = 0;
    bool at_origin = true;
    std::complex<double> t{0, 0};
    int J = 0;
    std::vector<double2> R, G, Glo, coef, pref;
    std::vector<double> norm, reflection;
    double2 self0{0, 0};
};

tcu_status lattice_setup_ck(int lsum, std::complex<double> k, const double* lat, size_t nk, const double* kpars,
                            double eta_in, const double* shift, LatticeSetupCk& S) {
    typedef std::complex<double> Z;
    if (lsum < 0 || lsum > LS_MAXL) return fail(TCU_INVALID_INPUT, "require 0 <= lmax_sum <= 14");
    if (!std::isfinite(k.real()) || !std::isfinite(k.imag()) || !(k.real() > 0.0) || k.imag() < 0.0 ||
        !(2.0 * k.imag() <= k.real()))
        return fail(TCU_INVALID_INPUT,
                    "the complex-wavenumber lattice sums take Re k > 0 and 0 <= Im k <= Re k / 2");
    if (!lat || !finite_all(lat, 4) || nk == 0 || !kpars || !finite_all(kpars, 2 * nk) || !shift ||
        !finite_all(shift, 3))
        return fail(TCU_INVALID_INPUT, "lattice, Bloch vectors and shift must be finite");
    const double a1x = lat[0], a1y = lat[1], a2x = lat[2], a2y = lat[3];
    const double det = a1x * a2y - a1y * a2x;
    S.area = std::fabs(det);
    if (!(S.area > 0.0) || !std::isfinite(S.area)) return fail(TCU_INVALID_INPUT, "lattice is numerically singular");
    double eta = eta_in;
    if (!std::isfinite(eta) || eta < 0.0) return fail(TCU_INVALID_INPUT, "the device lattice sums take a real split >= 0");
    const double kabs = std::abs(k);
    if (eta == 0.0) {  // lattice/cell.rs:164-175 with |k| (a real split)
        double kl = kabs * std::sqrt(S.area);
        eta = std::sqrt(2.0 * M_PI) / kl * std::max(kl / 8.0, 1.0);
    }
    // off the plane the split is capped at |k r_z eta| <= 1 where 1/(2 eta^2) <= 8 allows
    if (shift[2] != 0.0) eta = std::min(eta, std::max(0.25, 1.0 / (kabs * std::fabs(shift[2]))));
    const double c = 0.5 / (eta * eta);
    if (c > 8.0)
        return fail(TCU_INVALID_INPUT,
                    "Ewald split too small for the device lattice sums (require 1/(2 eta^2) <= 8); eta = 0 selects one");
    S.eta = eta;
    const double f0 = (a2y * shift[0] - a2x * shift[1]) / det, f1 = (-a1y * shift[0] + a1x * shift[1]) / det;
    const double c0 = std::round(f0), c1 = std::round(f1);
    S.R0x = c0 * a1x + c1 * a2x;
    S.R0y = c0 * a1y + c1 * a2y;
    S.sx = shift[0] - S.R0x;
    S.sy = shift[1] - S.R0y;
    S.sz = shift[2];
    S.at_origin = S.sx == 0.0 && S.sy == 0.0 && S.sz == 0.0;
    const Z ke = k * eta, ke2 = ke * ke;
    double zabs = 0.0;
    if (S.sz != 0.0) {
        const Z z = k * S.sz;
        zabs = std::abs(z);
        S.t = (z * eta) * (z * eta);
        if (!(std::abs(S.t) <= 16.0))
            return fail(TCU_INVALID_INPUT,
                        "shift too far off the lattice plane for the device lattice sums (require |k r_z eta|^2 <= 16)");
        double term = 1.0, big = 1.0, th = 0.5 * std::abs(S.t);
        int J = 1;
        for (; J < LS_TMAX; ++J) {
            term *= th / J;
            big = std::max(big, term);
            if (J > th && term < 1e-18 * big) break;
        }
        S.J = J;
    }
    // real space: Gaussian factor e^{-Re (k eta)^2 R^2/2 + c} below e^-46 times the polynomial growth
    const double decay = ke2.real();
    double Rc = std::sqrt(2.0 * (46.0 + c) / decay);
    for (int it = 0; it < 30; ++it)
        Rc = std::sqrt(2.0 * (46.0 + c + lsum * std::log(std::max(1.0, kabs * Rc)) +
                              (2 * lsum + 1) * std::log(std::max(1.0, eta))) /
                       decay);
    const double len1 = std::hypot(a1x, a1y), len2 = std::hypot(a2x, a2y);
    const double hdir = S.area / std::max(len1, len2);
    const double rin = std::hypot(S.sx, S.sy);
    long Nd = (long)std::ceil((Rc + rin) / hdir) + 1;
    if (Nd > 64) return fail(TCU_INVALID_INPUT, "lattice too elongated for the device lattice sums");
    for (long s = S.at_origin ? 1 : 0; s <= Nd; ++s)
        for (long n1 = -s; n1 <= s; ++n1)
            for (long n2 = -s; n2 <= s; ++n2) {
                if (std::max(std::labs(n1), std::labs(n2)) != s) continue;
                double x = n1 * a1x + n2 * a2x, y = n1 * a1y + n2 * a2y;
                if (std::hypot(x + S.sx, y + S.sy) <= Rc) S.R.push_back(make_double2(x, y));
            }
    // reciprocal: e^{-Re v} with Re v = (x2 - 1)/(2 eta^2), x2 = q.q Re(1/k^2), times the growth
    // |q/k|^lsum (2 eta^2)^n of the terms, e^(|t|/2) and the powers of |k r_z|, below e^-46
    const double b1x = 2 * M_PI * a2y / det, b1y = -2 * M_PI * a2x / det;
    const double b2x = -2 * M_PI * a1y / det, b2y = 2 * M_PI * a1x / det;
    const double rek2 = (1.0 / (k * k)).real();
    const double budget = 46.0 + 0.5 * std::abs(S.t) + lsum * std::log(std::max(1.0, zabs));
    double x2 = 1.0 + 2.0 * eta * eta * budget;
    for (int it = 0; it < 30; ++it)
        x2 = 1.0 + 2.0 * eta * eta *
                       (budget + 0.5 * lsum * std::log(std::max(1.0, x2 / (rek2 * kabs * kabs))) +
                        lsum * std::log(std::max(1.0, 2.0 * eta * eta)) + std::log(std::max(1.0, 1.0 / eta)));
    double kmax = 0.0;
    for (size_t i = 0; i < nk; ++i) kmax = std::max(kmax, std::hypot(kpars[2 * i], kpars[2 * i + 1]));
    const double qc = std::sqrt(x2 / rek2) + kmax;
    const double blen1 = std::hypot(b1x, b1y), blen2 = std::hypot(b2x, b2y);
    const double hrec = (4 * M_PI * M_PI / S.area) / std::max(blen1, blen2);
    long Nr = (long)std::ceil(qc / hrec) + 1;
    if (Nr > 64) return fail(TCU_INVALID_INPUT, "lattice or Bloch vectors out of range for the device lattice sums");
    DD bdd[2][2];
    reciprocal_dd(lat, bdd);
    for (long s = 0; s <= Nr; ++s)
        for (long n1 = -s; n1 <= s; ++n1)
            for (long n2 = -s; n2 <= s; ++n2) {
                if (std::max(std::labs(n1), std::labs(n2)) != s) continue;
                const DD x = dd_add(dd_mul(bdd[0][0], (double)n1), dd_mul(bdd[1][0], (double)n2));
                const DD y = dd_add(dd_mul(bdd[0][1], (double)n1), dd_mul(bdd[1][1], (double)n2));
                if (std::hypot(x.hi, y.hi) <= qc) {
                    S.G.push_back(make_double2(x.hi, y.hi));
                    S.Glo.push_back(make_double2(x.lo, y.lo));
                }
            }
    const int T = (lsum + 1) * (lsum + 1);
    S.norm.assign(T, 0.0);
    S.reflection.assign(T, 0.0);
    S.coef.assign((size_t)T * LS_PMAX * LS_FMAX, make_double2(0, 0));
    S.pref.assign(T, make_double2(0, 0));
    const Z mz = -k * S.sz, inv_k2 = 1.0 / (k * k);
    for (int l = 0; l <= lsum; ++l)
        for (int m = -l; m <= l; ++m) {
            const int lm = l * l + l + m, am = std::abs(m);
            S.norm[lm] = std::sqrt((2 * l + 1) / (4 * M_PI)) * std::exp(0.5 * (log_fact(l - m) - log_fact(l + m)));
            S.reflection[lm] = ((am % 2) ? -1.0 : 1.0) * std::exp(log_fact(l - am) - log_fact(l + am));
            // S_lmn (reciprocal.rs:22-60): coefficient of beta^(2p), p = (l-|m|-s)/2, order n:
            // (-k r_z)^(2n-s) / ((2n-s)! (s-n)! ((l+|m|-s)/2)! ((l-|m|-s)/2)!), n <= s <= min(l-|m|, 2n)
            for (int n = 0; n <= l - am; ++n)
                for (int sidx = n; sidx <= std::min(l - am, 2 * n); ++sidx) {
                    if ((l - am - sidx) % 2) continue;
                    const int zp = 2 * n - sidx, p = (l - am - sidx) / 2;
                    if (zp > 0 && S.sz == 0.0) continue;
                    const Z v = (zp == 0 ? Z(1.0, 0.0) : std::pow(mz, zp)) *
                                std::exp(-log_fact(zp) - log_fact(sidx - n) - log_fact(p + am) - log_fact(p));
                    S.coef[((size_t)lm * LS_PMAX + p) * LS_FMAX + n] = make_double2(v.real(), v.imag());
                }
            // sqrt(2l+1) (-i)^m sqrt((l+m)!(l-m)!) / (A k^2 (-2)^l)   (reciprocal.rs:320-330)
            const double mag = std::sqrt(2.0 * l + 1.0) * std::exp(0.5 * (log_fact(l + m) + log_fact(l - m))) /
                               (S.area * std::pow(-2.0, l));
            const int ph = ((m % 4) + 4) % 4;  // (-i)^m
            const Z mi(ph == 0 ? 1 : ph == 2 ? -1 : 0, ph == 1 ? -1 : ph == 3 ? 1 : 0);
            const Z pr = mag * mi * inv_k2;
            S.pref[lm] = make_double2(pr.real(), pr.imag());
        }
    {  // self term at l = 0 (reciprocal.rs:467-487): with a real split it does not depend on k
        double y = c, sum = 0.0, term = 1.0;
        for (int kk = 0; kk < 400; ++kk) {
            if (kk > 0) term *= y / kk;
            double add = term / (kk - 0.5);
            sum += add;
            if (kk > y && std::fabs(add) < 1e-18 * std::fabs(sum)) break;
        }
        double gre = -2.0 * std::sqrt(M_PI), gim = -sum / std::sqrt(y);
        double f = S.norm[0] * 0.5 / std::sqrt(M_PI);
        S.self0 = make_double2(f * gre, f * gim);
    }
    return TCU_OK;
}

}  // namespace

extern "C" tcu_status tcu_lsumsw2d_complex_batch(tcu_context* ctx, int lmax_sum, const double* k, const double* lattice,
                                                 size_t nk, const double* kpars, const double* shift, double eta,
                                                 double* out) {
    if (!ctx || !out || !k) return fail(TCU_INVALID_INPUT, "null context, wavenumber or output");
    std::lock_guard<std::recursive_mutex> lock(ctx->mu);
    cudaSetDevice(ctx->device);
    ProfGuard pg(ctx);
    const double zero[3] = {0.0, 0.0, 0.0};
    const std::complex<double> kc(k[0], k[1]);
    LatticeSetupCk S;
    tcu_status s = lattice_setup_ck(lmax_sum, kc, lattice, nk, kpars, eta, shift ? shift : zero, S);
    if (s) return s;
    const int T = (lmax_sum + 1) * (lmax_sum + 1);
    if (lattice_sum_ck_smem(lmax_sum, (int)S.R.size()) > 200 * 1024 || S.G.size() > (1u << 20))
        return fail(TCU_INVALID_INPUT, "lattice too elongated for the device lattice sums");
    Arena ar;
    size_t oK = ar.add(nk * 16), oO = ar.add(nk * T * 16), oR = ar.add(S.R.size() * 16), oG = ar.add(S.G.size() * 16),
           oN = ar.add(T * 8), oRf = ar.add(T * 8), oC = ar.add(S.coef.size() * 16), oP = ar.add(T * 16),
           oTab = ar.add(S.R.size() * T * 16), oGl = ar.add(S.Glo.size() * 16);
    DevBuf io(ctx);
    CK(io.alloc(ar.total), "lattice-sum buffers");
    void* b = io.p;
    cudaStream_t st = ctx->stream;
    CK(cudaMemcpyAsync(ar.at<void>(b, oK), kpars, nk * 16, cudaMemcpyHostToDevice, st), "copy");
    if (!S.R.empty())
        CK(cudaMemcpyAsync(ar.at<void>(b, oR), S.R.data(), S.R.size() * 16, cudaMemcpyHostToDevice, st), "copy");
    CK(cudaMemcpyAsync(ar.at<void>(b, oG), S.G.data(), S.G.size() * 16, cudaMemcpyHostToDevice, st), "copy");
    CK(cudaMemcpyAsync(ar.at<void>(b, oGl), S.Glo.data(), S.Glo.size() * 16, cudaMemcpyHostToDevice, st), "copy");
    CK(cudaMemcpyAsync(ar.at<void>(b, oN), S.norm.data(), T * 8, cudaMemcpyHostToDevice, st), "copy");
    CK(cudaMemcpyAsync(ar.at<void>(b, oRf), S.reflection.data(), T * 8, cudaMemcpyHostToDevice, st), "copy");
    CK(cudaMemcpyAsync(ar.at<void>(b, oC), S.coef.data(), S.coef.size() * 16, cudaMemcpyHostToDevice, st), "copy");
    CK(cudaMemcpyAsync(ar.at<void>(b, oP), S.pref.data(), T * 16, cudaMemcpyHostToDevice, st), "copy");
    CK(cudaMemsetAsync(ctx->d_status, 0, 4, st), "status");
    double2* tab = ar.at<double2>(b, oTab);
    const double2 kd = make_double2(k[0], k[1]);
    if (!S.R.empty()) {
        launch_real_table_ck(lmax_sum, kd, S.eta, (int)S.R.size(), ar.at<double2>(b, oR), S.sx, S.sy, S.sz,
                             ar.at<double>(b, oN), ar.at<double>(b, oRf), tab, st);
        ++ctx->launches;
    }
    LatticeSumCkArgs a;
    a.lsum = lmax_sum;
    a.k = kd;
    a.eta = S.eta;
    a.NR = (int)S.R.size();
    a.R = ar.at<double2>(b, oR);
    a.realtab = tab;
    a.NG = (int)S.G.size();
    a.G = ar.at<double2>(b, oG);
    a.Glo = ar.at<double2>(b, oGl);
    a.coef = ar.at<double2>(b, oC);
    a.pref = ar.at<double2>(b, oP);
    a.self0 = S.at_origin ? S.self0 : make_double2(0.0, 0.0);
    a.sx = S.sx;
    a.sy = S.sy;
    a.R0x = S.R0x;
    a.R0y = S.R0y;
    a.J = S.J;
    a.t = make_double2(S.t.real(), S.t.imag());
    const std::complex<double> ksq = kc * kc;
    a.ksq = make_double2(ksq.real(), ksq.imag());
    // the outgoing sheets of the split (lattice/sheets.rs): arg (k eta)^2 = arg k^2 for a real eta
    a.turn = std::arg(ksq);
    const double angle = std::fabs(a.turn) + 0.5;
    a.has_near = angle < M_PI / 2 ? 1 : 0;
    a.near = a.has_near ? std::pow(std::tan(angle), 2) : 0.0;
    a.nk = (int)nk;
    a.kpar = ar.at<double2>(b, oK);
    a.out = ar.at<double2>(b, oO);
    a.ldo = T;
    a.status = ctx->d_status;
    launch_lattice_sum_ck(a, (int)std::min<size_t>(nk, 148 * 8), st);
    ++ctx->launches;
    int stw = 0;
    CK(cudaMemcpyAsync(&stw, ctx->d_status, sizeof(int), cudaMemcpyDeviceToHost, st), "status");
    if ((s = sync_status(ctx, "lattice sums"))) return s;
    if (stw == 9)
        return fail(TCU_INVALID_INPUT, "lattice sum is at a diffraction threshold; supply a limiting complex wavenumber");
    if (stw) return fail(TCU_DEVICE_ERROR, "lattice sums: device status " + std::to_string(stw));
    CK(cudaMemcpyAsync(out, ar.at<void>(b, oO), nk * T * 16, cudaMemcpyDeviceToHost, st), "copy");
    return sync_status(ctx, "lattice sums");
}

extern "C" tcu_status tcu_array_solve_batch(tcu_context* ctx, int lmax, double k0, double radius, const double* eps,
                                            const double* lattice, size_t nk, const double* kpars, double eta,
                                            double* out) {
    if (!ctx || !out || !kpars || nk == 0) return fail(TCU_INVALID_INPUT, "null context, Bloch vectors or output");
    std::lock_guard<std::recursive_mutex> lock(ctx->mu);
    cudaSetDevice(ctx->device);
    ProfGuard pg(ctx);
    if (lmax < 1 || lmax > 6) return fail(TCU_INVALID_INPUT, "the batched array solve takes 1 <= lmax <= 6");
    const size_t M = 2 * (size_t)lmax * (lmax + 2);
    Arena ar;
    size_t oK = ar.add(nk * 16), oX = ar.add(nk * M * M * 16);
    DevBuf io(ctx);
    CK(io.alloc(ar.total), "array-solve buffers");
    CK(cudaMemcpyAsync(ar.at<void>(io.p, oK), kpars, nk * 16, cudaMemcpyHostToDevice, ctx->stream), "copy");
    tcu_status s = array_solve_device(ctx, lmax, k0, radius, eps, lattice, nk, ar.at<double2>(io.p, oK), eta, kpars,
                                      ar.at<double2>(io.p, oX));
    if (s) return s;
    CK(cudaMemcpyAsync(out, ar.at<void>(io.p, oX), nk * M * M * 16, cudaMemcpyDeviceToHost, ctx->stream), "copy");
    return sync_status(ctx, "periodic array solve");
}

extern "C" tcu_status tcu_context_set_learned_weights(tcu_context* ctx, double reach_diameters, size_t count,
                                                      const double* weights) {
    if (!ctx || !std::isfinite(reach_diameters) || reach_diameters > 20.0 || (count > 0 && !weights) ||
        (count > 0 && !finite_all(weights, count)))
        return fail(TCU_INVALID_INPUT, "require reach <= 20 diameters and finite weights");
    std::lock_guard<std::recursive_mutex> lock(ctx->mu);
    ctx->precond_reach = reach_diameters > 0.0 ? reach_diameters : -1.0;
    ctx->learned_weights.assign(weights, weights + count);
    return TCU_OK;
}

extern "C" size_t tcu_learned_weight_count(int lmax) {
    return lmax >= 1 && lmax <= 7 ? (size_t)learned_weight_count(lmax) : 0;
}

struct tcu_learned_problem {
    tcu_context* ctx = nullptr;
    int L = 0;
    size_t N = 0, n = 0;
    int nprobe = 0;
    double* d_pos = nullptr;
    cplx* d_T = nullptr;
    cplx* d_V = nullptr;
    LearnedProblem lp;
    ~tcu_learned_problem() {
        for (void* q : {(void*)d_pos, (void*)d_T, (void*)d_V})
            if (q) ctx->pool.free(q);
    }
};

extern "C" tcu_status tcu_learned_problem_create(tcu_context* ctx, int lmax, double k0, size_t N, const double* radii,
                                                 const double* eps, const double* positions, int nprobe,
                                                 const double* V, tcu_learned_problem** out) {
    if (!ctx || !out || !V || nprobe <= 0 || nprobe > 64 || lmax < 1 || lmax > 7)
        return fail(TCU_INVALID_INPUT,
                    "require a context, an output handle, 1 <= lmax <= 7 and 1 <= nprobe <= 64 probe vectors");
    *out = nullptr;
    std::lock_guard<std::recursive_mutex> lock(ctx->mu);
    ProfGuard pg(ctx);
    CK(cudaSetDevice(ctx->device), "device");
    tcu_status s = validate_spheres(lmax, k0, N, radii, eps, positions);
    if (s) return s;
    const DevPlan* P;
    if ((s = get_plan(ctx, lmax, &P))) return s;
    const size_t n = N * 2 * (size_t)lmax * (lmax + 2);
    if (!finite_all(V, 2 * n * (size_t)nprobe)) return fail(TCU_INVALID_INPUT, "probe vectors must be finite");
    auto p = std::make_unique<tcu_learned_problem>();
    p->ctx = ctx;
    p->L = lmax;
    p->N = N;
    p->n = n;
    p->nprobe = nprobe;
    if ((s = dev_alloc(ctx, &p->d_pos, 3 * N, "positions")) || (s = dev_alloc(ctx, &p->d_T, N * lmax * 4, "T blocks")) ||
        (s = dev_alloc(ctx, &p->d_V, n * nprobe, "probes")))
        return s;
    DevBuf tmp(ctx);
    Arena ga;
    const size_t o_r = ga.add(N * 8), o_e = ga.add(N * 16);
    CK(tmp.alloc(ga.total), "geometry");
    double* d_r = ga.at<double>(tmp.p, o_r);
    cplx* d_e = ga.at<cplx>(tmp.p, o_e);
    CK(cudaMemcpyAsync(p->d_pos, positions, N * 24, cudaMemcpyHostToDevice, ctx->stream), "copy");
    CK(cudaMemcpyAsync(d_r, radii, N * 8, cudaMemcpyHostToDevice, ctx->stream), "copy");
    CK(cudaMemcpyAsync(d_e, eps, N * 16, cudaMemcpyHostToDevice, ctx->stream), "copy");
    CK(cudaMemcpyAsync(p->d_V, V, n * nprobe * 16, cudaMemcpyHostToDevice, ctx->stream), "copy");
    CK(cudaMemsetAsync(ctx->d_status, 0, 4, ctx->stream), "status");
    launch_mie(lmax, k0, (int)N, d_r, d_e, p->d_T, ctx->d_status, ctx->stream);
    ++ctx->launches;
    if ((s = read_status(ctx, "Mie coefficients"))) return s;
    std::unique_ptr<CoarseSolve> coarse;
    // the training loss differentiates through a fixed linear preconditioner: always a factor
    if ((s = make_coarse(ctx, k0, N, radii, eps, positions, &coarse, true)))
        return fail(s, std::string("coarse dipole system: ") + g_last_error);
    s = p->lp.build(ctx->stream, *P, lmax, (int)N, k0, p->d_pos, positions, radii, eps, p->d_T, ctx->precond_reach,
                    nprobe, p->d_V, std::move(coarse), &ctx->launches);
    if (s == TCU_OUT_OF_MEMORY) return fail(s, "training problem: out of device memory");
    if (s) return fail(s, "training problem: device failure");
    *out = p.release();
    return TCU_OK;
}

extern "C" tcu_status tcu_learned_problem_loss_grad(tcu_learned_problem* p, const double* weights, double* loss,
                                                    double* grad) {
    if (!p || !weights || !loss || !grad) return fail(TCU_INVALID_INPUT, "null argument");
    const size_t nw = (size_t)learned_weight_count(p->L);
    if (!finite_all(weights, nw)) return fail(TCU_INVALID_INPUT, "weights must be finite");
    std::lock_guard<std::recursive_mutex> lock(p->ctx->mu);
    ProfGuard pg(p->ctx);
    CK(cudaSetDevice(p->ctx->device), "device");
    tcu_status s = p->lp.loss_grad(weights, loss, grad, p->ctx->stream);
    if (s) return fail(s, "training problem: device failure");
    return TCU_OK;
}

extern "C" tcu_status tcu_learned_problem_probes(tcu_learned_problem* p, double* out) {
    if (!p || !out) return fail(TCU_INVALID_INPUT, "null argument");
    std::lock_guard<std::recursive_mutex> lock(p->ctx->mu);
    CK(cudaSetDevice(p->ctx->device), "device");
    tcu_status s = p->lp.probes((double2*)out, p->ctx->stream);
    if (s) return fail(s, "training problem: device failure");
    return TCU_OK;
}

extern "C" tcu_status tcu_learned_problem_destroy(tcu_learned_problem* p) {
    if (!p) return TCU_OK;
    tcu_context* ctx = p->ctx;
    std::lock_guard<std::recursive_mutex> lock(ctx->mu);
    cudaSetDevice(ctx->device);
    cudaStreamSynchronize(ctx->stream);
    delete p;
    return TCU_OK;
}

extern "C" tcu_status tcu_batch_solve(tcu_context* ctx, size_t count, const tcu_cluster_desc* clusters, int precision,
                                      int* order) {
    if (!ctx || (count > 0 && !clusters)) return fail(TCU_INVALID_INPUT, "null context or cluster list");
    if (precision < TCU_FP64 || precision > TCU_AUTO) return fail(TCU_INVALID_INPUT, "unknown precision");
    std::vector<size_t> idx(count);
    for (size_t i = 0; i < count; ++i) {
        const tcu_cluster_desc& c = clusters[i];
        if (c.lmax < 1 || c.lmax > 10 || !c.B || !c.X || c.p <= 0)
            return fail(TCU_INVALID_INPUT, "cluster " + std::to_string(i) + ": invalid lmax, incidence or output");
        idx[i] = i;
    }
    auto modes = [&](size_t i) { return clusters[i].N * 2 * (size_t)clusters[i].lmax * (clusters[i].lmax + 2); };
    std::stable_sort(idx.begin(), idx.end(), [&](size_t a, size_t b) { return modes(a) > modes(b); });
    for (size_t q = 0; q < count && order; ++q) order[q] = (int)idx[q];
    auto solve_one = [&](tcu_context* c_ctx, size_t i) -> tcu_status {
        const tcu_cluster_desc& c = clusters[i];
        int prec = precision == TCU_AUTO ? (modes(i) >= ctx->auto_crossover ? TCU_MIXED : TCU_FP64) : precision;
        tcu_factor* f = nullptr;
        tcu_status s = tcu_sphere_cluster_factor(c_ctx, c.lmax, c.k0, c.N, c.radii, c.eps, c.positions, prec, &f);
        if (s == TCU_OK) {
            s = tcu_factor_solve(f, c.B, c.p, c.X, c.certificates);
            tcu_factor_destroy(f);
        }
        return s;
    };
    const int K = (int)std::min<size_t>((size_t)batch_workers(), count);
    if (K <= 1) {
        for (size_t q = 0; q < count; ++q) {
            tcu_status s = solve_one(ctx, idx[q]);
            if (s) return fail(s, "cluster " + std::to_string(idx[q]) + ": " + g_last_error);
        }
        return TCU_OK;
    }
    // K host threads, each with its own context (stream, scratch, pooled allocator), take the
    // clusters largest first from a shared counter: the latency-bound panels and sweeps of
    // different clusters overlap on the GPU.
    {
        std::lock_guard<std::recursive_mutex> lock(ctx->mu);
        while ((int)ctx->workers.size() < K) {
            tcu_context* w = nullptr;
            tcu_status s = tcu_context_create(ctx->device, &w);
            if (s) return s;
            ctx->workers.push_back(w);
        }
    }
    std::vector<long long> fb0(K), ln0(K);
    for (int w = 0; w < K; ++w) {
        tcu_context* wc = ctx->workers[w];
        wc->refine_target = ctx->refine_target;
        // 192 rows per panel CTA: panels of up to ~28,000 rows on 148 CTAs, and the panels of
        // smaller clusters on few enough SMs that the workers' panels run side by side (64
        // clusters of the sweep: 3.70 s with 32 rows, 3.03 s with 200 rows, 4 workers)
        wc->panel_rows = 192;
        wc->fallback_above = ctx->fallback_above;
        fb0[w] = wc->fallbacks;
        ln0[w] = wc->launches;
    }
    std::atomic<size_t> next{0};
    std::atomic<bool> stop{false};
    std::mutex emu;
    tcu_status first = TCU_OK;
    std::string msg;
    std::vector<std::thread> threads;
    for (int w = 0; w < K; ++w)
        threads.emplace_back([&, w] {
            cudaSetDevice(ctx->device);
            while (!stop.load()) {
                const size_t q = next.fetch_add(1);
                if (q >= count) break;
                const tcu_status s = solve_one(ctx->workers[w], idx[q]);
                if (s) {
                    std::lock_guard<std::mutex> g(emu);
                    if (first == TCU_OK) {
                        first = s;
                        msg = "cluster " + std::to_string(idx[q]) + ": " + g_last_error;
                    }
                    stop = true;
                }
            }
        });
    for (auto& t : threads) t.join();
    for (int w = 0; w < K; ++w) {
        ctx->fallbacks += ctx->workers[w]->fallbacks - fb0[w];
        ctx->launches += ctx->workers[w]->launches - ln0[w];
    }
    if (first) return fail(first, msg);
    return TCU_OK;
}

// Precision autotuner of the batched solves: times assembly + factorization + one refined
// solve in FP64 and in mixed precision on synthetic clusters (spheres of radius 0.2 on a
// jittered cubic grid of spacing 0.55, eps 2.25 + 0.01i, k0 2, lmax 4) of growing size, and
// sets the crossover of TCU_AUTO to the smallest size from which the mixed path is faster
// (and stays faster on the larger sizes). sizes: 0..count-1 unknown counts written out with
// their times (ms), may be NULL.
extern "C" tcu_status tcu_context_autotune(tcu_context* ctx, size_t* crossover, int count, size_t* sizes,
                                           double* ms_fp64, double* ms_mixed) {
    if (!ctx) return fail(TCU_INVALID_INPUT, "null context");
    std::lock_guard<std::recursive_mutex> lock(ctx->mu);
    CK(cudaSetDevice(ctx->device), "device");
    const int spheres[] = {8, 16, 32, 64, 128, 192};
    const int ns = sizeof(spheres) / sizeof(spheres[0]);
    std::vector<double> tf(ns), tm(ns);
    std::vector<size_t> nn(ns);
    cudaEvent_t e0, e1;
    CK(cudaEventCreate(&e0), "event");
    CK(cudaEventCreate(&e1), "event");
    tcu_status s = TCU_OK;
    for (int q = 0; q < ns && !s; ++q) {
        const int N = spheres[q];
        const int side = (int)std::ceil(std::cbrt((double)N));
        std::vector<double> r(N, 0.2), eps(2 * N), pos(3 * N);
        uint64_t st = 0x9E3779B97F4A7C15ull * (q + 1);
        for (int i = 0; i < N; ++i) {
            eps[2 * i] = 2.25;
            eps[2 * i + 1] = 0.01;
            const int a = i % side, b = (i / side) % side, c = i / (side * side);
            const int idx[3] = {a, b, c};
            for (int d = 0; d < 3; ++d) {
                st = st * 6364136223846793005ull + 1442695040888963407ull;
                const double jitter = ((st >> 11) * (1.0 / 9007199254740992.0) - 0.5) * 0.1;
                pos[3 * i + d] = 0.55 * idx[d] + jitter;
            }
        }
        nn[q] = (size_t)N * 48;
        std::vector<double> B(2 * nn[q], 0.0), X(2 * nn[q]);
        for (size_t j = 0; j < nn[q]; ++j) B[2 * j] = 1.0 / (1.0 + j % 7);
        for (int prec = 0; prec < 2 && !s; ++prec) {
            float best = 1e30f;
            for (int rep = 0; rep < 2 && !s; ++rep) {
                tcu_factor* f = nullptr;
                cudaEventRecord(e0, ctx->stream);
                s = tcu_sphere_cluster_factor(ctx, 4, 2.0, N, r.data(), eps.data(), pos.data(),
                                              prec ? TCU_MIXED : TCU_FP64, &f);
                if (!s) s = tcu_factor_solve(f, B.data(), 1, X.data(), nullptr);
                cudaEventRecord(e1, ctx->stream);
                cudaEventSynchronize(e1);
                float ms = 0.f;
                cudaEventElapsedTime(&ms, e0, e1);
                best = std::min(best, ms);
                if (f) tcu_factor_destroy(f);
            }
            (prec ? tm : tf)[q] = best;
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (s) return s;
    size_t cross = nn[ns - 1] + 1;
    for (int q = ns - 1; q >= 0 && tm[q] < tf[q]; --q) cross = nn[q];
    ctx->auto_crossover = cross;
    if (crossover) *crossover = cross;
    for (int q = 0; q < count && q < ns; ++q) {
        if (sizes) sizes[q] = nn[q];
        if (ms_fp64) ms_fp64[q] = tf[q];
        if (ms_mixed) ms_mixed[q] = tm[q];
    }
    return TCU_OK;
}

extern "C" tcu_status tcu_context_wait_selftest(tcu_context* ctx, double limit_seconds) {
    if (!ctx || !std::isfinite(limit_seconds) || limit_seconds < 0.0)
        return fail(TCU_INVALID_INPUT, "require a context and a finite limit >= 0");
    std::lock_guard<std::recursive_mutex> lock(ctx->mu);
    DevBuf bar(ctx);
    CK(bar.alloc(sizeof(unsigned) * 4), "self-test barrier");
    CK(cudaMemsetAsync(bar.p, 0, sizeof(unsigned) * 4, ctx->stream), "self-test barrier");
    CK(cudaMemsetAsync(ctx->d_status, 0, sizeof(int), ctx->stream), "self-test status");
    launch_barrier_selftest((unsigned*)bar.p, ctx->d_status, limit_seconds, ctx->stream);
    ctx->launches += 1;
    tcu_status s = read_status(ctx, "bounded-wait self-test");
    CK(cudaMemsetAsync(ctx->d_status, 0, sizeof(int), ctx->stream), "self-test status");
    tcu_status s2 = sync_status(ctx, "bounded-wait self-test");
    if (s == TCU_OK) return fail(TCU_DEVICE_ERROR, "bounded-wait self-test: the barrier passed with an arrival missing");
    return s2 ? s2 : s;
}

extern "C" tcu_status tcu_context_set_refinement(tcu_context* ctx, double target, double fallback_above) {
    if (!ctx || !(target > 0.0) || !(fallback_above > 0.0) || !std::isfinite(target) || !std::isfinite(fallback_above))
        return fail(TCU_INVALID_INPUT, "require positive finite refinement tolerances");
    std::lock_guard<std::recursive_mutex> lock(ctx->mu);
    ctx->refine_target = target;
    ctx->fallback_above = fallback_above;
    return TCU_OK;
}
