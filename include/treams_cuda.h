/* treams_cuda.h — C ABI of the B200 (sm_100a) cluster multiple-scattering library.
 *
 * Every entry point replaces one Rust function of treams-core on the cluster hot path
 * (cited per declaration as path:line inside the treams-rs tree). Complex numbers are
 * two doubles (re, im), the layout of num_complex::Complex64; matrices are column-major,
 * as nalgebra's DMatrix. Host-pointer entry points copy in and out; `_dev` entry points
 * take device pointers and run on the context's stream.
 *
 * Errors: every call returns a tcu_status. The first six codes mirror treams-core's
 * Error variants (lib.rs:384-411); the message of the last failure on the calling thread
 * is tcu_last_error_message(). No call aborts or traps.
 *
 * Threading: a context owns one CUDA stream and its workspaces. Calls on one context are
 * serialised by an internal mutex; distinct contexts may be used concurrently. Results
 * do not depend on timing: every reduction runs in a fixed order.
 */
#ifndef TREAMS_CUDA_H
#define TREAMS_CUDA_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum tcu_status {
    TCU_OK = 0,
    TCU_INVALID_INPUT = 1,      /* Error::InvalidInput */
    TCU_SPECIAL_FUNCTION = 2,   /* Error::SpecialFunction */
    TCU_NON_FINITE = 3,         /* Error::NonFinite */
    TCU_NOT_CONVERGED = 4,      /* Error::NotConverged */
    TCU_SINGULAR = 5,           /* Error::Singular */
    TCU_OUT_OF_MEMORY = 6,      /* Error::OutOfMemory */
    TCU_DEVICE_ERROR = 7,       /* CUDA runtime or kernel failure */
    TCU_TIMEOUT = 8             /* a bounded device-side wait gave up */
} tcu_status;

typedef enum tcu_precision {
    TCU_FP64 = 0,   /* complex128 LU, FP64 DMMA trailing updates */
    TCU_MIXED = 1,  /* complex64 LU, 3-pass split tcgen05 updates (FP16 or TF32 pieces), FP64 refinement */
    TCU_AUTO = 2    /* batch solves only: per cluster, MIXED from the context's crossover on (2048 modes
                       until tcu_context_autotune measures it), else FP64 */
} tcu_precision;

typedef enum tcu_preconditioner {
    TCU_PRECOND_NONE = 0,          /* plain GMRES on I - T C */
    TCU_PRECOND_BLOCK_JACOBI = 1,  /* block Jacobi over nearest-neighbour sphere groups (<= 96 modes) */
    TCU_PRECOND_LEARNED = 2,       /* coarse dipole solve + near field weighted by the trained graph network */
    TCU_PRECOND_TWO_LEVEL = 3      /* coarse dipole solve + unweighted near field (the method without the network) */
} tcu_preconditioner;

typedef struct tcu_context tcu_context;
typedef struct tcu_factor tcu_factor;

/* Convergence certificate of one right-hand side (linalg/gmres.rs:86-93): the residual
 * b - A x is recomputed in FP64 from the returned x. */
typedef struct tcu_certificate {
    int iterations;          /* GMRES iterations or refinement sweeps */
    double residual_norm;    /* ||T b - (I - T C) x||_2 */
    double rhs_norm;         /* ||T b||_2 */
} tcu_certificate;

/* GMRES options (linalg/gmres.rs:22-79). */
typedef struct tcu_gmres_options {
    double rtol;
    double atol;
    int restart;
    int max_iterations;
} tcu_gmres_options;

/* ---- context ------------------------------------------------------------------------ */
tcu_status tcu_context_create(int device, tcu_context** out);
/* Destroys the context and every factor still alive on it (their handles become invalid). */
tcu_status tcu_context_destroy(tcu_context* ctx);
/* The CUDA stream (cudaStream_t) the context runs on, for callers with device pointers. */
void* tcu_context_stream(tcu_context* ctx);
/* Thread-local message of the last failed call on this thread ("" if none). */
const char* tcu_last_error_message(void);
/* Number of kernel launches the context has issued (a counter for benchmarks). */
long long tcu_context_launches(tcu_context* ctx);
/* Refinement tolerances of tcu_factor_solve on this context (no counterpart in the reference):
 * sweeps stop at ||r|| <= target ||T b|| (default 1e-13); a mixed solve left above
 * fallback_above ||T b|| (default 1e-12) is finished with an FP64 factor. */
tcu_status tcu_context_set_refinement(tcu_context* ctx, double target, double fallback_above);
/* Number of mixed-precision solves whose FP64 refinement stalled above the fallback tolerance
 * and that were finished by a second factor (TF32 pieces, then FP64) of the same cluster. */
long long tcu_context_fallbacks(tcu_context* ctx);
/* Precision autotuner of batched solves (no counterpart in the reference): times assembly +
 * factorization + one refined solve in FP64 and in mixed precision on synthetic lmax-4 clusters
 * of 384 to 9216 unknowns and sets TCU_AUTO's crossover to the smallest size from which the
 * mixed path stays faster. crossover (may be NULL) receives it; the first count sizes and times
 * (ms) go to sizes, ms_fp64, ms_mixed (each may be NULL). Takes about a second. */
tcu_status tcu_context_autotune(tcu_context* ctx, size_t* crossover, int count, size_t* sizes, double* ms_fp64,
                                double* ms_mixed);
/* Failure-detection self-test (no counterpart in the reference): runs the LU panel's grid
 * barrier with one arrival missing, so that its bounded wait gives up after limit_seconds
 * (clamped to [0, 4] s). Returns TCU_TIMEOUT, as a factorization whose CTAs never meet
 * would, and leaves the context usable; any other status means the wait did not give up. */
tcu_status tcu_context_wait_selftest(tcu_context* ctx, double limit_seconds);
/* Per-stage device timing with CUDA events on the context stream (off by default).
 * Stages: 0 assembly, 1 LU panel, 2 row swaps, 3 triangular block (TRSM), 4 trailing
 * update GEMM, 5 operand packing, 6 triangular solves, 7 matrix-free operator, 8 Mie,
 * 9 lattice sums, 10 batched small LU, 11 dipole blocks of the two-level preconditioner,
 * 12 its near-field term. Reading synchronises the stream. */
tcu_status tcu_context_set_profiling(tcu_context* ctx, int enabled);
tcu_status tcu_context_stage_time(tcu_context* ctx, int stage, long long* launches, double* total_ms);
tcu_status tcu_context_reset_stage_times(tcu_context* ctx);

/* ---- translation coefficients -------------------------------------------------------- */
/* M x M block (M = 2 lmax (lmax + 2)) of vector spherical wave translation coefficients
 * from a source to a destination at displacement disp = destination - source, helicity
 * (helicity != 0) or parity modes, outgoing (singular != 0) or regular radial functions;
 * column-major, source modes outer. Replaces TranslationPlan::evaluate (sw/plan.rs:282). */
tcu_status tcu_translation_block(tcu_context* ctx, int lmax, double k, const double* disp, int singular,
                                 int helicity, double* out);

/* Translation coefficients of single mode pairs at complex polar arguments, the elementwise
 * sw.translate (python/treams_rs/sw.py:70; treams-core sw/polar.rs:251 polar_translation_array).
 * labels: count x 6 ints (lambda, mu, pol of the destination mode, l, m, qol of the source
 * mode; degrees 1..10); args: count x 3 complex (kr, theta, phi of k (r_destination -
 * r_source)); out: count complex. helicity != 0: A + (2 pol - 1) B for pol == qol, else 0;
 * parity: A for pol == qol, else B. singular != 0 expands an outgoing wave (0 at kr = 0). */
tcu_status tcu_translate(tcu_context* ctx, size_t count, const int* labels, const double* args, int helicity,
                         int singular, double* out);
/* Wigner 3j symbol (j1 j2 j3; m1 m2 m3) (special/wigner.rs:263 wigner3j), degrees <= 60,
 * by Racah's closed formula in binary128 on the host (no device work, no context). */
double tcu_wigner3j(int j1, int j2, int j3, int m1, int m2, int m3);

/* ---- Mie T and incident fields -------------------------------------------------------- */
/* 2 x 2 Mie blocks in mode order, lmax per sphere, N spheres: out N * lmax * 4 complex,
 * row-major per block (tmatrix/sphere.rs:43-80, coeffs/mie.rs:209). */
tcu_status tcu_mie_blocks(tcu_context* ctx, int lmax, double k0, size_t N, const double* radii, const double* eps,
                          double* out);

/* Regular expansion of p plane waves at the N sphere positions (pw/expand.rs:308-360):
 * kvecs holds 3 complex per wave, pols 0/1 per wave (helicity); out n x p column-major. */
tcu_status tcu_plane_wave_expansion(tcu_context* ctx, int lmax, size_t N, const double* positions, int p,
                                    const double* kvecs, const int* pols, double* out);

/* Scattering and extinction cross sections of p columns (python/treams_rs/_tmatrix.py:
 * 413-441, flux 0.5): sca = Re(x^H O x) / k0^2 with O the regular coupling between all
 * positions (applied matrix-free), ext = -Re(b^H x) / k0^2. */
tcu_status tcu_cross_sections(tcu_context* ctx, int lmax, double k0, size_t N, const double* positions, int p,
                              const double* x, const double* b, double* sca, double* ext);

/* ---- dense cluster solve ------------------------------------------------------------- */
/* Assemble I - T C for N spheres (eps: N complex, positions: 3 N doubles) and factor it
 * in the given precision. Replaces cluster::sphere_cluster_factor (cluster/spheres.rs:85)
 * = cluster_parts + InteractionFactor::from_blocks (cluster/interaction.rs:194). */
tcu_status tcu_sphere_cluster_factor(tcu_context* ctx, int lmax, double k0, size_t N, const double* radii,
                                     const double* eps, const double* positions, int precision, tcu_factor** out);
/* Device-pointer variant: radii, eps, positions are device arrays. */
tcu_status tcu_sphere_cluster_factor_dev(tcu_context* ctx, int lmax, double k0, size_t N, const double* radii,
                                         const double* eps, const double* positions, int precision,
                                         tcu_factor** out);
/* Solve (I - T C) X = T B for p incident columns B (n x p), X out (n x p); certificates
 * (p entries) may be NULL. Replaces InteractionFactor::solve (cluster/interaction.rs:214).
 * The solve refines in FP64 until ||r|| <= 1e-13 ||T b|| (at most 10 sweeps on mixed factors, 2 on
 * FP64 factors, stopping when a sweep does not halve the residual); if a mixed solve is left
 * with ||r|| > 1e-12 ||T b||, it is finished with a second factor of the same cluster, made once
 * and kept: a mixed one with TF32 pieces after FP16 pieces, an FP64 one after TF32 pieces
 * (tcu_context_fallbacks counts these solves). */
tcu_status tcu_factor_solve(tcu_factor* f, const double* B, int p, double* X, tcu_certificate* certificates);
tcu_status tcu_factor_solve_dev(tcu_factor* f, const double* B, int p, double* X, tcu_certificate* certificates);
/* Interacting T-matrix X = (I - T C)^-1 T of the cluster (n x n, column-major, host), the
 * solution for every column of the block-diagonal T (cluster::interaction,
 * cluster/interaction.rs:292-315), refined in FP64 like tcu_factor_solve. */
tcu_status tcu_factor_interacting_tmatrix(tcu_factor* f, double* X);
/* T-matrix of the whole cluster in one spherical basis of degree lmax_global (<= 10) at origin:
 * sum_ij R(origin <- r_i) X_ij R(r_j <- origin) with regular translations (the cluster's
 * expand into a global basis, python/treams_rs/_operators.py:183 expand), Mg x Mg column-major
 * (Mg = 2 lmax_global (lmax_global + 2)). Valid for scatterers outside a sphere around origin
 * that holds all the spheres' centres. */
tcu_status tcu_factor_global_tmatrix(tcu_factor* f, int lmax_global, const double* origin, double* out);
/* Adjoint solve Y = (I - T C)^-H G with the factor (linalg/mod.rs:436 solve_adjoint_in_place),
 * refined in FP64 against the matrix-free adjoint operator like tcu_factor_solve; certificates
 * report ||G - (I - T C)^H Y|| and ||G||. No counterpart as a public call in the reference. */
tcu_status tcu_factor_solve_adjoint(tcu_factor* f, const double* G, int p, double* Y, tcu_certificate* certificates);
/* Gradient of incident columns for the factor: out = T^H (I - T C)^-H G
 * (InteractionFactor::pullback_incident, cluster/interaction.rs:221-227). */
tcu_status tcu_factor_pullback_incident(tcu_factor* f, const double* G, int p, double* out,
                                        tcu_certificate* certificates);
/* Dimension n = N M of a factor. */
size_t tcu_factor_dimension(const tcu_factor* f);
tcu_status tcu_factor_destroy(tcu_factor* f);

/* One cluster of a batch: geometry and materials (host arrays as for
 * tcu_sphere_cluster_factor), p incident columns B (n x p) and the solution X (n x p). */
typedef struct tcu_cluster_desc {
    int lmax;
    double k0;
    size_t N;
    const double* radii;
    const double* eps;
    const double* positions;
    const double* B;
    int p;
    double* X;
    tcu_certificate* certificates; /* p entries, or NULL */
} tcu_cluster_desc;

/* Solve a batch of independent clusters (no counterpart in the reference, which solves one
 * cluster per call): largest first (n = N * 2 lmax (lmax + 2)), each assembled, factored,
 * solved and released. TCU_BATCH_WORKERS (default 4) host threads with one stream each take
 * the clusters from a shared queue, so the latency-bound stages of different clusters overlap
 * and device memory holds at most that many operators at a time. precision: TCU_FP64,
 * TCU_MIXED or TCU_AUTO. order (count entries, may be NULL) receives the dispatch order (size
 * order). Stops at the first failing cluster; the message names it. */
tcu_status tcu_batch_solve(tcu_context* ctx, size_t count, const tcu_cluster_desc* clusters, int precision,
                           int* order);

/* The assembled operator I - T C (n x n complex128, column-major, host), for inspection. */
tcu_status tcu_cluster_operator(tcu_context* ctx, int lmax, double k0, size_t N, const double* radii,
                                const double* eps, const double* positions, double* out);

/* ---- matrix-free cluster ------------------------------------------------------------- */
/* y = (I - T C) x for p columns without forming C (cluster/iterative.rs:225-232). */
tcu_status tcu_cluster_apply(tcu_context* ctx, int lmax, double k0, size_t N, const double* radii, const double* eps,
                             const double* positions, int p, const double* x, double* y);
/* Allocation-free y = (I - T C) x (no counterpart in the reference; for callers that cannot
 * allocate device memory, e.g. inside another framework's memory plan). Every pointer is a
 * device pointer (radii N doubles, eps N complex, positions 3 N doubles, x and y n x p
 * complex); the call runs on `stream` (a cudaStream_t, may be NULL) and needs no context.
 * Scratch (plan tables, Mie blocks, a status word) lives in one 8 MiB static device array
 * per GPU: the plan plus N * lmax * 64 bytes must fit, larger clusters are rejected with
 * TCU_INVALID_INPUT. The first call on a device looks up that array's address. Calls that
 * overlap on the GPU race on the shared array. The call copies from pageable host memory and
 * synchronises `stream` (geometry check and status read), so it cannot be used under stream
 * capture. Errors: tcu_last_error_message(). */
tcu_status tcu_cluster_apply_noalloc(void* stream, int lmax, double k0, size_t N, const double* radii,
                                     const double* eps, const double* positions, int p, const double* x, double* y);
/* Restarted GMRES on (I - T C) X = T B (cluster/iterative.rs:264-284, linalg/gmres.rs:119).
 * The preconditioner, if any, is applied on the right; certificates report the true
 * unpreconditioned residual. For lmax 2..5 the harmonic tables of all N (N - 1) sphere pairs
 * are built once per call and kept in device memory for the operator applications
 * (N^2 (2 lmax + 1)^2 16 bytes: 14 GB at 4096 spheres and lmax 3), and the two-level
 * preconditioners store those of their dipole blocks too; each set only while it takes at most
 * half of the free device memory, else the tables are rebuilt per application (the results
 * agree to rounding). The environment variable TCU_APPLY=fly turns the stored tables off. */
tcu_status tcu_iterative_solve(tcu_context* ctx, int lmax, double k0, size_t N, const double* radii,
                               const double* eps, const double* positions, const double* B, int p,
                               const tcu_gmres_options* options, int preconditioner, double* X,
                               tcu_certificate* certificates);

/* Incident-field gradient of the matrix-free cluster: out = T^H Y with Y = (I - T C)^-H G from
 * one unpreconditioned adjoint GMRES solve per column (IterativeSphereCluster::pullback,
 * cluster/iterative.rs:460-488, its `incident` part; the position, radius and permittivity
 * gradients of that call are not built). Certificates report the adjoint GMRES residuals. */
tcu_status tcu_iterative_pullback_incident(tcu_context* ctx, int lmax, double k0, size_t N, const double* radii,
                                           const double* eps, const double* positions, const double* G, int p,
                                           const tcu_gmres_options* options, double* out,
                                           tcu_certificate* certificates);

/* Preconditioners TCU_PRECOND_LEARNED and TCU_PRECOND_TWO_LEVEL (no counterpart in the
 * reference, whose iterative solver is unpreconditioned): right preconditioner
 *   z = P A_cc^-1 v_c + (I + T C_near^Theta)(v - A P A_cc^-1 v_c)
 * with A_cc = I - T_1 C_11 the cluster's dipole (l = 1) system, factored once by this
 * library's dense LU, P its injection into the full mode space, and C_near^Theta the
 * translation blocks of the sphere pairs closer than the reach, every (degree, degree)
 * sub-block of pair (i, j) scaled by Theta_ij. TWO_LEVEL uses Theta = 1; LEARNED predicts Theta
 * with a graph network over the pairs (node features of each sphere, edge features of each
 * pair; 2 lmax^2 real outputs per edge). */
/* Near-field reach in sphere diameters (<= 0: the compiled-in 3) and network weights
 * (count 0: the compiled-in weights of the lmax solved; a count that does not match
 * tcu_learned_weight_count of that lmax uses Theta = 1). */
tcu_status tcu_context_set_learned_weights(tcu_context* ctx, double reach_diameters, size_t count,
                                           const double* weights);
/* Number of network weights for lmax (0 outside 1..7). */
size_t tcu_learned_weight_count(int lmax);

/* Training of the network on the GPU (no counterpart in the reference). A training problem
 * holds one cluster (host arrays as for tcu_sphere_cluster_factor) and nprobe probe vectors V
 * (n x nprobe complex, column-major, host; 1 <= nprobe <= 64), turned into coarse-corrected
 * unit-norm probes r1 = (v - A P A_cc^-1 v_c) / ||.||. loss_grad evaluates, on the device,
 * loss = sum_p ||r1_p - A M_Theta r1_p||^2 (M_Theta r = r + T C_near^Theta r, A = I - T C in FP64)
 * and its gradient in every weight (forward and backward kernels of the network; the gradient
 * through Theta uses the adjoint operator A^H). probes copies the r1 to the host. */
typedef struct tcu_learned_problem tcu_learned_problem;
tcu_status tcu_learned_problem_create(tcu_context* ctx, int lmax, double k0, size_t N, const double* radii,
                                      const double* eps, const double* positions, int nprobe, const double* V,
                                      tcu_learned_problem** out);
tcu_status tcu_learned_problem_loss_grad(tcu_learned_problem* p, const double* weights, double* loss, double* grad);
tcu_status tcu_learned_problem_probes(tcu_learned_problem* p, double* out);
tcu_status tcu_learned_problem_destroy(tcu_learned_problem* p);

/* ---- 2D lattice sums and periodic arrays --------------------------------------------- */
/* Ewald lattice sums D_lm (lattice/mod.rs:11-15, 283; ewald.rs:39-270) of a 2D lattice
 * for nk Bloch vectors, every degree l <= lmax_sum and order m (table index l*l+l+m):
 * k real wavenumber, lattice 2 x 2 row vectors, kpars nk x 2, shift r[3] = 0 (one sphere
 * per cell), eta (0 = automatic split, cell.rs:164-175). out nk x (lmax_sum+1)^2. */
tcu_status tcu_lsumsw2d_batch(tcu_context* ctx, int lmax_sum, double k, const double* lattice, size_t nk,
                              const double* kpars, double eta, double* out);
/* The same at a shift r (lattice::sum with shift, lattice/mod.rs:283): D_lm(k, kpar, r) =
 * sum'_R h_l(k|r+R|) Y_lm(-r-R) e^{i kpar.R}, the in-plane part of r reduced into the cell on
 * the host (lattice/ewald.rs:610-665). Off the lattice plane (r[2] != 0) the reciprocal part
 * takes every order of S_lmn and the t-series of F_(1/2-n)(v, t) (lattice/reciprocal.rs:22-60,
 * lattice/reduced.rs:223) with the split capped at |k r_z eta| <= 1 down to eta = 1/4 (the sum does
 * not depend on it); shifts with (k r_z eta)^2 > 16 at that split are rejected (TCU_INVALID_INPUT). */
tcu_status tcu_lsumsw2d_shift_batch(tcu_context* ctx, int lmax_sum, double k, const double* lattice, size_t nk,
                                    const double* kpars, const double* shift, double eta, double* out);
/* The same sums at a complex wavenumber k = k[0] + i k[1] (a lossy embedding; lattice::sum takes
 * a complex k, lattice/mod.rs:283): Re k > 0, 0 <= Im k <= Re k / 2, any shift r[3] (null: r = 0),
 * a real split eta (0: the automatic split of cell.rs:164-175 taken at |k|). Each diffraction
 * order is evaluated on its outgoing sheet (lattice/sheets.rs). out nk x (lmax_sum+1)^2. */
tcu_status tcu_lsumsw2d_complex_batch(tcu_context* ctx, int lmax_sum, const double* k, const double* lattice,
                                      size_t nk, const double* kpars, const double* shift, double eta, double* out);
/* Periodic array of one sphere per cell: X(kpar) = (I - T S(kpar))^-1 T for nk Bloch
 * vectors (cluster/interaction.rs:292 with sw::lattice_expansion, sw/expansion.rs:418).
 * out nk x M x M (column-major per kpar). */
tcu_status tcu_array_solve_batch(tcu_context* ctx, int lmax, double k0, double radius, const double* eps,
                                 const double* lattice, size_t nk, const double* kpars, double eta, double* out);

#ifdef __cplusplus
}
#endif

#endif /* TREAMS_CUDA_H */
