"""Cluster-solve throughput on one B200 per rank.

Workload: the 512-sphere, lmax-4 precision cluster (n = 24,576 unknowns, three plane-wave
incidences), seeded synthetic geometry. One step = assemble I - T C, factor it and solve
the three columns to an FP64 residual <= 1e-13 |T b| (relative error well below 1e-10):
`tcu_sphere_cluster_factor_dev` + `tcu_factor_solve_dev`. The headline is the mixed
path (complex64 LU with split-TF32 tensor-core trailing updates + FP64 refinement); the
same run then times the plain FP64 drop-in on the same inputs (`fp64` and
`speedup_vs_fp64` in the JSON line, `--no-compare` skips it) beside two library yardsticks
(cuSOLVER zgetrf through torch.linalg.lu_factor on the same complex128 operator, and the
cuBLAS FP64/complex128 GEMM rate that serves as the FP64 roofline). `--precision fp64`
makes the FP64 path the headline.

value: solves/s with inputs resident in HBM, device-timed with CUDA events on the library
stream (max over ranks). e2e: the same through the host-buffer C ABI with host<->device
copies inside the timed region. The matrix (4.8-9.7 GB) is far larger than L2, so no
flush is needed. cpu_baseline (rank 0, N = 1) and `--impl reference` solve the full
512-sphere cluster on the host cores with the CPU restatement (C++ oracle assembly of
I - T C + LAPACK zgetrf/zgetrs): no sample, no extrapolation; the main line also states the
relative difference between the GPU solution and that CPU solution.
"""
from __future__ import annotations

import argparse
import json
import os
import pathlib
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = pathlib.Path(__file__).resolve().parent
for p in (ROOT, ROOT / "treams-rs_b200"):
    if str(p) not in sys.path:
        sys.path.insert(0, str(p))

import numpy as np  # noqa: E402

METRIC = "cluster-solve/s, 512 spheres lmax 4: mixed+learned vs plain FP64 @1e-10 err"
UNIT = "solves/s"


# DRAM traffic of the trailing-update kernel relative to its algorithmic bytes (the
# complex64 C block read and written once, 16 m^2 bytes), from an ncu capture of the
# m = 11,776 launch of a 256-sphere solve: 2.395 GB measured for 2.219 GB algorithmic.
# Traffic grows with m^2 like the algorithmic bytes, so the bench scales this ratio to the
# average launch of the measured workload.
TF32_TRAFFIC = {"ratio": 2.275 / 2.219,
                "note": "dram__bytes_read.sum + dram__bytes_write.sum of tf32_update_kernel per launch: "
                        "ncu ratio to algorithmic bytes (1.03, two-pass m=11776 launch of a 256-sphere solve) "
                        "x the average algorithmic bytes (complex64 C read + write) of this workload's "
                        "update launches, paired K = 256 updates included"}


def update_launch_shapes(n: int, nb: int, pairs: bool = True) -> list:
    """(rows, columns) of every trailing-update launch of the mixed LU, in the order the library
    runs them: with pairs, panel a updates panel b's columns, panel b its own block rows, then
    one update with both panels."""
    out, pend = [], False
    for k0 in range(0, n, nb):
        w = min(nb, n - k0)
        cols = n - k0 - w
        if cols <= 0:
            break
        if pend:
            out += [(w, cols), (cols, cols)]
            pend = False
        elif pairs and cols > nb:
            out.append((cols, nb))
            pend = True
        else:
            out.append((cols, cols))
    return out


def update_launch_bytes(n: int, nb: int, pairs: bool = True) -> float:
    """Average algorithmic bytes (complex64 C read + write) per trailing-update launch."""
    shapes = update_launch_shapes(n, nb, pairs)
    return sum(16.0 * m * c for m, c in shapes) / len(shapes)


# Peaks measured on this pool's B200s (STREAM-style copy, cuBLAS bf16 GEMM as a burst and as a
# seconds-long loop under the power cap); used when MEASURED_PEAKS.json is absent.
POOL_PEAKS = {"hbm_gbs": 6540.0, "bf16_tflops": 1605.2, "bf16_tflops_sustained": 1371.8}


def peaks():
    try:
        d = json.loads((ROOT / "MEASURED_PEAKS.json").read_text())
        d.setdefault("source", "MEASURED_PEAKS.json")
        return d
    except Exception:
        return dict(POOL_PEAKS, source="pool measurement recorded in bench.py")


class Clocks:
    """nvidia-smi clock samples during the timed region."""

    def __init__(self, index: int):
        self.proc = None
        fd, name = tempfile.mkstemp(prefix="treams_clocks_", suffix=".csv")
        os.close(fd)
        self.path = pathlib.Path(name)
        try:
            self.fh = open(self.path, "w")
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={index}", "--query-gpu=index,clocks.sm,clocks.max.sm,power.draw,"
                 "clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
                 "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
                 "clocks_event_reasons.sw_power_cap", "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=self.fh, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self) -> dict:
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        self.proc.wait()
        self.fh.close()
        text = self.path.read_text()
        self.path.unlink(missing_ok=True)
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in text.splitlines():
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for name, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons)}


def lu_update_flops(n: int, nb: int) -> float:
    """Useful real flops of all trailing updates of a right-looking complex LU (8 per MAC)."""
    total = 0.0
    for k0 in range(0, n, nb):
        w = min(nb, n - k0)
        m = n - k0 - w
        total += 8.0 * m * m * w
    return total


def cpu_full_solve(spheres: int = 512) -> dict:
    """One full solve of the precision cluster on the host cores: the CPU restatement's FP64
    assembly of I - T C (C++ oracle, OpenMP) and LAPACK zgetrf + zgetrs of the three columns
    (scipy's OpenBLAS, all threads), no sample and no extrapolation. Returns the timing and
    the solution X."""
    import oracle
    import scipy.linalg
    from treams_b200 import workloads

    w = workloads.precision_cluster(count=spheres)
    t0 = time.perf_counter()
    A, tb = oracle.cluster_operator(w.lmax, w.k0, w.radii, w.eps, w.positions)
    t1 = time.perf_counter()
    B = oracle.plane_wave_expansion(w.lmax, w.positions, w.kvecs, w.pols)
    TB = oracle.apply_t(w.lmax, tb, B)
    lu, piv = scipy.linalg.lu_factor(A, overwrite_a=True, check_finite=False)
    X = scipy.linalg.lu_solve((lu, piv), TB, check_finite=False)
    t2 = time.perf_counter()
    del A, lu
    return {"seconds": t2 - t0, "assembly_s": t1 - t0, "lu_solve_s": t2 - t1, "X": X, "n": w.n}


def cpu_threads() -> int:
    try:
        return len(os.sched_getaffinity(0))
    except Exception:
        return os.cpu_count() or 1


def cpu_baseline_line(spheres: int) -> tuple[dict, np.ndarray]:
    r = cpu_full_solve(spheres)
    line = {"value": 1.0 / r["seconds"], "unit": UNIT, "cores": cpu_threads(), "kind": "port",
            "sample": f"the full workload, no extrapolation: {spheres} spheres lmax 4 (n={r['n']}), 3 plane waves; "
                      "C++ restatement FP64 assembly (OpenMP) + LAPACK zgetrf/zgetrs (OpenBLAS), one solve",
            "seconds_per_solve": r["seconds"], "assembly_s": r["assembly_s"], "lu_solve_s": r["lu_solve_s"]}
    return line, r["X"]


def _timed(stream, fn):
    """Device time (CUDA events on the library stream) and wall time of one call."""
    import torch

    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    t0 = time.perf_counter()
    e0.record(stream)
    out = fn()
    e1.record(stream)
    torch.cuda.synchronize()
    return out, e0.elapsed_time(e1), (time.perf_counter() - t0) * 1e3


def iterative_workload(ctx, stream, count: int = 4096, with_cpu: bool = True, c128_peak=None) -> dict:
    """The 4096-sphere lmax-3 matrix-free cluster (n = 122,880): GMRES(50) to 1e-8 without,
    with block-Jacobi and with the learned preconditioner (set-up included). GMRES applies the
    operator from the pair tables stored once per solve (14 GB here)."""
    import treams_b200 as t
    from treams_b200 import workloads

    w = workloads.learned_cluster(count=count)
    c = t.SphereCluster(w.lmax, w.k0, w.radii, w.eps, w.positions, ctx=ctx)
    B = t.plane_wave_expansion(w.lmax, w.positions, w.kvecs, w.pols, ctx=ctx)[:, 0]
    out = {"workload": f"{count} spheres r 0.2, 20% fill, eps 4+0.05i, k0 1.5, lmax 3 (n={w.n}); GMRES(50) to 1e-8",
           "unit": "solves/s", "warmup": "one untimed solve of each kind first; ms = the faster of two timed solves"}
    kinds = ("none", "block_jacobi", "two_level", "learned")
    for kind in kinds:  # first-use costs (module loading, plan, allocations) stay out of the timing
        c.solve(B, rtol=1e-8, restart=50, max_iterations=600, preconditioner=kind)
    for kind in kinds:  # the faster of two timed solves: the set-up runs partly on the host cores
        runs = [_timed(stream, lambda: c.solve(B, rtol=1e-8, restart=50, max_iterations=600, preconditioner=kind))
                for _ in range(2)]
        sol, ms, wall = min(runs, key=lambda r: r[1])
        cert = sol.convergence[0]
        out[kind] = {"iterations": cert.iterations, "rel_residual": cert.residual_norm / cert.rhs_norm,
                     "ms": ms, "value": 1e3 / ms}
    out["iteration_ratio_block_jacobi_over_learned"] = out["block_jacobi"]["iterations"] / out["learned"]["iterations"]
    out["time_ratio_block_jacobi_over_learned"] = out["block_jacobi"]["ms"] / out["learned"]["ms"]
    out["iteration_ratio_two_level_over_learned"] = out["two_level"]["iterations"] / out["learned"]["iterations"]
    out["note"] = ("two_level: coarse dipole solve (inner GMRES on the 6N dipole system above 6144 dipole modes, "
                   "else its dense LU) + near-field Neumann term; learned: the same with the graph network's "
                   "near-field weights (Theta = 1 while no trained weights beat it); set-up included in ms; "
                   "the operator and the two dipole blocks from harmonic tables stored once per solve")
    # the stored-table application: device stage time of (tables + 1 application) and of
    # (tables + 3 applications) through the ABI with TCU_APPLY=stored
    stage = {}
    os.environ["TCU_APPLY"] = "stored"
    try:
        for nc in (1, 3):
            xs = np.random.default_rng(nc).standard_normal((w.n, nc)) + 0j
            c.apply(xs)
            ctx.reset_stage_times()
            ctx.set_profiling(True)
            c.apply(xs)
            ctx.set_profiling(False)
            stage[nc] = ctx.stage_times().get("apply", (0, 0.0))[1]
    finally:
        os.environ.pop("TCU_APPLY", None)
    per = (stage[3] - stage[1]) / 2.0
    pairs = w.radii.size * (w.radii.size - 1)
    flops = 8.0 * pairs * (2 * w.lmax + 1) ** 2 * 2 * w.lmax * (w.lmax + 2)
    tf = flops / (per / 1e3) / 1e12 if per > 0 else None
    out["stored_operator"] = {
        "ms_per_application": per, "table_build_ms": stage[1] - per,
        "table_bytes": pairs * (2 * w.lmax + 1) ** 2 * 16,
        "roofline": {"bound": "fp64 tensor (DMMA)", "achieved": tf, "peak": c128_peak, "unit": "TFLOP/s",
                     "frac": tf / c128_peak if tf and c128_peak else None,
                     "note": "8 (2L+1)^2 2L(L+2) useful flops per ordered pair (complex products of the table "
                             "matrix with the coefficients); peak: measured cuBLAS complex128 GEMM rate (of measured)"}}
    # one matrix-free operator application: device time and the CPU restatement on the host cores
    x = np.ones((w.n, 1), complex)
    _, ms_apply, _ = _timed(stream, lambda: c.apply(x))
    if with_cpu:
        import oracle
        t0 = time.perf_counter()
        oracle.iterative_apply(w.lmax, w.k0, w.radii, w.eps, w.positions, x)
        sec = time.perf_counter() - t0
        out["matvec"] = {"gpu_e2e_ms": ms_apply,
                         "cpu_baseline": {"value": 1.0 / sec, "unit": "matvecs/s", "cores": cpu_threads(),
                                          "kind": "port", "sample": f"one full matvec (I - T C) x of the {count}-sphere "
                                                                    "cluster, C++ restatement (OpenMP)"}}
    return out


def periodic_workload(ctx, stream, nk: int = 4096, with_cpu: bool = True, fp64_peak=None) -> dict:
    """The periodic array: square lattice (period 0.54), one sphere per cell (r 0.2, eps 9),
    k0 4, lmax 6, 4096 Bloch vectors: lattice sums (degrees <= 12) and X = (I - T S)^-1 T."""
    from treams_b200 import lattice as tl
    from treams_b200 import workloads

    w = workloads.periodic_array(nk=nk)
    tl.array_solve_batch(w.lmax, w.k0, w.radius, w.eps, w.lattice, w.kpars[:8], ctx=ctx)  # warm-up
    # the same Bloch vectors at a shift off the lattice plane, and in a lossy embedding (complex k)
    shift = (0.1 * w.period, 0.2 * w.period, 0.3 * w.period)
    tl.lsumsw2d_batch(12, w.k0 * (1 + 0.05j), w.lattice, w.kpars[:8], shift=shift, ctx=ctx)  # warm-up
    _, ms_off, _ = _timed(stream, lambda: tl.lsumsw2d_batch(12, w.k0, w.lattice, w.kpars, shift=shift, ctx=ctx))
    _, ms_ck, _ = _timed(stream, lambda: tl.lsumsw2d_batch(12, w.k0 * (1 + 0.05j), w.lattice, w.kpars, shift=shift,
                                                           ctx=ctx))
    ctx.reset_stage_times()
    ctx.set_profiling(True)
    _, ms_sums, _ = _timed(stream, lambda: tl.lsumsw2d_batch(12, w.k0, w.lattice, w.kpars, ctx=ctx))
    _, ms_all, _ = _timed(stream, lambda: tl.array_solve_batch(w.lmax, w.k0, w.radius, w.eps, w.lattice, w.kpars,
                                                               ctx=ctx))
    ctx.set_profiling(False)
    st = ctx.stage_times()
    nk = len(w.kpars)
    lu_ms = st.get("small_lu", (0, 0.0))[1]
    flops = nk * 8.0 * 96 ** 3
    out = {"workload": f"periodic array: period {w.period:.4f}, lmax 6, {nk} Bloch vectors", "unit": "kpar/s",
           "lattice_sums_e2e_ms": ms_sums, "array_solve_e2e_ms": ms_all,
           "lattice_sums_off_plane_e2e_ms": ms_off, "lattice_sums_complex_k_off_plane_e2e_ms": ms_ck,
           "lattice_sums_variants": "degrees <= 12 at the shift (0.1, 0.2, 0.3) periods, real k0 and k0 (1 + 0.05i)",
           "array_solve_e2e_value": nk / (ms_all / 1e3),
           "stages_ms": {k: v[1] for k, v in st.items()},
           "array_kernel_fp64_tflops": flops / (lu_ms / 1e3) / 1e12 if lu_ms else None,
           "array_kernel_roofline": {"bound": "fp64", "peak": fp64_peak, "unit": "TFLOP/s",
                                     "frac": (flops / (lu_ms / 1e3) / 1e12) / fp64_peak if lu_ms and fp64_peak
                                     else None,
                                     "note": "8 M^3 real flops per Bloch vector (Gauss-Jordan inversion of the "
                                             "M = 96 operator) over the small-LU stage; peak = measured cuBLAS "
                                             "float64 GEMM rate (of measured)"},
           "note": "e2e includes the host copies of X (nk x 96 x 96 complex, 604 MB)"}
    if with_cpu:
        import oracle
        sample = 64
        t0 = time.perf_counter()
        for kp in w.kpars[:sample]:
            oracle.array_solve(w.lmax, w.k0, w.radius, w.eps, w.lattice, kp)
        sec = time.perf_counter() - t0
        out["cpu_baseline"] = {"value": sample / sec, "unit": "kpar/s", "cores": 1, "kind": "port",
                               "sample": f"the first {sample} of the {nk} Bloch vectors: lattice sums (binary128 "
                                         "restatement) + 96 x 96 array solve each, one thread"}
    return out


def batch_workload(ctx, stream, count: int, with_cpu: bool = True) -> dict:
    """Clusters 0..count-1 of the 256-cluster heterogeneous sweep (N ~ U{16..256}, lmax ~
    U{3..6}, k0 ~ U[0.5, 3]; one plane wave each) in one tcu_batch_solve call, precision auto.
    The roofline counts the useful LU flops (8/3) n^3 of every cluster."""
    import treams_b200 as t
    from treams_b200 import workloads

    batch, modes, flops = [], 0, 0.0
    for c in range(count):
        w = workloads.batch_cluster(c)
        B = t.plane_wave_expansion(w.lmax, w.positions, w.kvecs, w.pols, ctx=ctx)
        batch.append((w.lmax, w.k0, w.radii, w.eps, w.positions, B))
        modes += w.n
        flops += 8.0 / 3.0 * float(w.n) ** 3
    tuned = ctx.autotune()  # the FP64/mixed crossover of "auto", measured on this GPU
    t.batch_solve(batch[:2], "auto", ctx=ctx)  # warm-up
    fb0 = ctx.fallbacks
    (X, certs, order), ms, wall = _timed(stream, lambda: t.batch_solve(batch, "auto", ctx=ctx))
    worst = max(c[0].residual_norm / c[0].rhs_norm for c in certs)
    out = {"workload": f"clusters 0..{count - 1} of the 256-cluster sweep ({modes} unknowns in total)",
           "unit": "clusters/s", "value": count / (ms / 1e3), "ms": ms, "max_rel_residual": worst,
           "fp64_fallbacks": ctx.fallbacks - fb0,
           "precision": f"auto (mixed from {tuned['crossover']} unknowns, else fp64; autotuned)", "autotune": tuned,
           "useful_lu_tflops": flops / (ms / 1e3) / 1e12}
    if with_cpu:
        import oracle
        import scipy.linalg
        sample = 4
        t0 = time.perf_counter()
        for lmax, k0, r, e, x, B in batch[:sample]:
            A, tb = oracle.cluster_operator(lmax, k0, r, e, x)
            scipy.linalg.lu_solve(scipy.linalg.lu_factor(A, overwrite_a=True, check_finite=False),
                                  oracle.apply_t(lmax, tb, B), check_finite=False)
        sec = time.perf_counter() - t0
        out["cpu_baseline"] = {"value": sample / sec, "unit": "clusters/s", "cores": cpu_threads(), "kind": "port",
                               "sample": f"clusters 0..{sample - 1} of the sweep: C++ restatement assembly + LAPACK "
                                         "zgetrf/zgetrs, all host threads"}
    return out


def fp64_yardsticks(w, ctx, dev) -> dict:
    """Library yardsticks for the FP64 arm on the same complex128 operator: cuSOLVER zgetrf +
    zgetrs through torch.linalg.lu_factor / lu_solve (cuSOLVER forced), and the cuBLAS GEMM
    rates (float64 and complex128, 8192^2, 8 real flops per complex MAC) that bound the FP64
    trailing update. Comparison only; the product path never calls them."""
    import torch
    import treams_b200 as t

    def timed(fn, reps):
        fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(reps):
            out = fn()
        e1.record()
        torch.cuda.synchronize()
        return out, e0.elapsed_time(e1) / reps

    res = {}
    for name, dt, mult in (("fp64", torch.float64, 2.0), ("c128", torch.complex128, 8.0)):
        a = torch.randn(8192, 8192, dtype=dt, device=dev)
        b = torch.randn(8192, 8192, dtype=dt, device=dev)
        _, ms = timed(lambda: a @ b, 5)
        res[f"cublas_{name}_gemm_tflops"] = mult * 8192.0 ** 3 / (ms / 1e3) / 1e12
        del a, b
    torch.backends.cuda.preferred_linalg_library("cusolver")
    A_h = t.cluster_operator(w.lmax, w.k0, w.radii, w.eps, w.positions, ctx=ctx)  # column-major complex128
    A = torch.from_numpy(A_h).to(dev)  # keeps the column-major strides
    del A_h
    rhs = torch.randn(A.shape[0], 3, dtype=torch.complex128, device=dev)
    (LU, piv), ms_f = timed(lambda: torch.linalg.lu_factor(A), 2)
    _, ms_s = timed(lambda: torch.linalg.lu_solve(LU, piv, rhs), 3)
    res.update({"cusolver_zgetrf_ms": ms_f, "cusolver_zgetrs_ms": ms_s,
                "cusolver_zgetrf_tflops": 8.0 / 3.0 * float(A.shape[0]) ** 3 / (ms_f / 1e3) / 1e12,
                "note": "torch.linalg.lu_factor/lu_solve with preferred_linalg_library('cusolver') on the "
                        "library-assembled complex128 operator (9.66 GB)"})
    del A, LU, piv, rhs
    torch.cuda.empty_cache()
    return res


def workload_config(spheres: int) -> dict:
    """The `config` of both arms (identical, so the two lines describe the same workload)."""
    return {"workload": f"precision cluster: {spheres} spheres lmax 4 (n={48 * spheres}), 3 plane waves, seed 1002",
            "l2": "inputs larger than L2 (matrix 4.8-9.7 GB), no flush"}


def run_reference(args, rank: int, world: int) -> None:
    """The reference arm: full solves of the workload on the host cores with the CPU
    restatement (no GPU work). A full solve takes minutes of CPU time, so at most
    --reference-max-steps of them are timed and no warm-up solve is run; the line states the
    steps it ran beside the steps it was asked for."""
    if rank != 0:
        return
    steps = max(1, min(args.steps, args.reference_max_steps))
    samples = [cpu_full_solve(args.spheres)["seconds"] for _ in range(steps)]
    sec = float(np.mean(samples))
    v = 1.0 / sec
    threads = cpu_threads()
    sample = (f"the full workload, no extrapolation: {args.spheres} spheres lmax 4 (n={48 * args.spheres}); C++ "
              "restatement FP64 assembly (OpenMP) + LAPACK zgetrf/zgetrs (OpenBLAS), all host threads")
    line = {"metric": METRIC, "value": v, "unit": UNIT, "impl": "reference", "n_gpus": world, "steps": steps,
            "warmup": 0, "steps_requested": args.steps, "warmup_requested": args.warmup,
            "ms_per_step": sec * 1e3, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "c128", "data": "synthetic", "precision": "fp64 (CPU restatement + LAPACK)",
            "parallelism": "rank 0 only", "config": workload_config(args.spheres),
            "cpu_baseline": {"value": v, "unit": UNIT, "cores": threads, "kind": "port", "sample": sample},
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--precision", default="mixed", choices=["mixed", "fp64"])
    ap.add_argument("--spheres", type=int, default=512)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-compare", dest="compare", action="store_false",
                    help="skip the plain FP64 comparison arm of the mixed headline")
    ap.add_argument("--compare-steps", type=int, default=3)
    ap.add_argument("--no-e2e", action="store_true", help="skip the host-buffer end-to-end timing (profiling runs)")
    ap.add_argument("--no-extras", dest="extras", action="store_false",
                    help="skip the 4096-sphere GMRES and the periodic-array workloads")
    ap.add_argument("--iterative-spheres", type=int, default=4096)
    ap.add_argument("--periodic-kpars", type=int, default=4096)
    ap.add_argument("--batch-clusters", type=int, default=256,
                    help="clusters of the 256-cluster heterogeneous sweep timed in the batch workload")
    ap.add_argument("--reference-max-steps", type=int, default=1,
                    help="full CPU solves timed by --impl reference (each takes minutes)")
    args = ap.parse_args()

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dist = None
    if world > 1:
        import torch.distributed as dist_mod
        from datetime import timedelta

        dist = dist_mod
        backend = "gloo" if args.impl == "reference" else "nccl"
        if backend == "nccl":
            import torch
            torch.cuda.set_device(local)
        dist.init_process_group(backend, timeout=timedelta(seconds=600))

    if args.impl == "reference":
        run_reference(args, rank, world)
        if dist:
            dist.destroy_process_group()
        return

    import torch
    import treams_b200 as t
    from treams_b200 import _lib, workloads

    torch.cuda.set_device(local)
    ctx = t.Context(local)
    lib = _lib.lib()
    stream = torch.cuda.ExternalStream(ctx.stream)
    w = workloads.precision_cluster(count=args.spheres)
    dev = torch.device("cuda", local)

    def barrier():
        if dist:
            dist.barrier()

    def reduce_max(vals):
        if not dist:
            return vals
        tt = torch.tensor(vals, dtype=torch.float64, device=dev)
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        return [float(v) for v in tt]

    def measure(precision, steps, warmup, with_e2e, fp64_peak=None):
        return _measure_impl(args, precision, steps, warmup, with_e2e, ctx=ctx, lib=lib, stream=stream, w=w,
                             dev=dev, world=world, local=local, dist=dist, barrier=barrier, reduce_max=reduce_max,
                             fp64_peak=fp64_peak)

    head = measure(args.precision, args.steps, args.warmup, not args.no_e2e)
    with_cpu = world == 1 and rank == 0 and not args.no_cpu_baseline
    other, yard = None, None
    if args.compare and args.precision == "mixed":
        yard = fp64_yardsticks(w, ctx, dev)
    extras = {}
    if args.extras:
        fp64_peak = yard["cublas_fp64_gemm_tflops"] if yard else None
        extras["iterative"] = iterative_workload(ctx, stream, args.iterative_spheres, with_cpu,
                                                 yard["cublas_c128_gemm_tflops"] if yard else None)
        extras["periodic"] = periodic_workload(ctx, stream, args.periodic_kpars, with_cpu, fp64_peak)
        extras["batch"] = batch_workload(ctx, stream, args.batch_clusters, with_cpu)
    if yard is not None:
        other = measure("fp64", min(args.steps, args.compare_steps), 1, False,
                        fp64_peak=yard["cublas_c128_gemm_tflops"])
    if rank == 0:
        line = head["line"]
        if other is not None:
            o = other["line"]
            asm = o["stages_ms_per_step"].get("assemble", 0.0)
            cus_ms = asm + yard["cusolver_zgetrf_ms"] + yard["cusolver_zgetrs_ms"]
            yard["cusolver_step_ms"] = cus_ms
            yard["cusolver_step_note"] = "this library's FP64 assembly + cuSOLVER zgetrf + zgetrs (3 columns)"
            line["fp64"] = {"value": o["value"], "ms_per_step": o["ms_per_step"], "steps": o["steps"],
                            "warmup": o["warmup"], "max_rel_residual": o["max_rel_residual"],
                            "roofline": o["roofline"], "stages_ms_per_step": o["stages_ms_per_step"],
                            "gpu_launches": o["gpu_launches"], "yardsticks": yard}
            line["speedup_vs_fp64"] = line["value"] / o["value"]
            best = max(o["value"], 1e3 / cus_ms)
            line["speedup_vs_best_fp64"] = line["value"] / best
            line["best_fp64"] = "this library" if o["value"] >= 1e3 / cus_ms else "cuSOLVER zgetrf"
        line.update(extras)
        if with_cpu:
            cpu, Xc = cpu_baseline_line(args.spheres)
            Xg = head["X"]
            errs = [float(np.linalg.norm(Xg[:, c] - Xc[:, c]) / np.linalg.norm(Xc[:, c])) for c in range(Xc.shape[1])]
            cpu["max_rel_diff_gpu_vs_cpu"] = max(errs)
            line["cpu_baseline"] = cpu
        print(json.dumps(line), flush=True)
    ctx.close()
    if dist:
        dist.destroy_process_group()


def _measure_impl(args, precision, steps, warmup, with_e2e, *, ctx, lib, stream, w, dev, world, local, dist,
                  barrier, reduce_max, fp64_peak=None):
    import ctypes

    import torch
    import treams_b200 as t
    from treams_b200 import _lib

    prec = t.MIXED if precision == "mixed" else t.FP64
    r_d = torch.tensor(w.radii, dtype=torch.float64, device=dev)
    e_d = torch.view_as_real(torch.tensor(w.eps, dtype=torch.complex128, device=dev)).contiguous()
    x_d = torch.tensor(w.positions, dtype=torch.float64, device=dev).contiguous()
    B_h = t.plane_wave_expansion(w.lmax, w.positions, w.kvecs, w.pols, ctx=ctx)  # (n, p) F-order
    p = B_h.shape[1]
    B_d = torch.tensor(np.asfortranarray(B_h).ravel(order="F"), dtype=torch.complex128, device=dev)
    X_d = torch.zeros_like(B_d)
    n = B_h.shape[0]
    certs = (_lib.Certificate * p)()
    torch.cuda.synchronize()

    def step_device():
        h = _lib.P()
        _lib._check(lib.tcu_sphere_cluster_factor_dev(ctx.handle, w.lmax, w.k0, w.radii.size, r_d.data_ptr(),
                                                      e_d.data_ptr(), x_d.data_ptr(), prec, ctypes.byref(h)))
        _lib._check(lib.tcu_factor_solve_dev(h, B_d.data_ptr(), p, X_d.data_ptr(), certs))
        lib.tcu_factor_destroy(h)

    radii_h = np.ascontiguousarray(w.radii)
    eps_h = np.ascontiguousarray(w.eps)
    pos_h = np.ascontiguousarray(w.positions)
    B_pin = torch.from_numpy(np.asfortranarray(B_h).ravel(order="F")).pin_memory()
    X_pin = torch.zeros_like(B_pin).pin_memory()
    h2d = radii_h.nbytes + eps_h.nbytes + pos_h.nbytes + B_pin.numel() * 16
    d2h = X_pin.numel() * 16

    def step_host():
        h = _lib.P()
        _lib._check(lib.tcu_sphere_cluster_factor(ctx.handle, w.lmax, w.k0, w.radii.size, radii_h.ctypes.data,
                                                  eps_h.ctypes.data, pos_h.ctypes.data, prec, ctypes.byref(h)))
        _lib._check(lib.tcu_factor_solve(h, B_pin.data_ptr(), p, X_pin.data_ptr(), certs))
        lib.tcu_factor_destroy(h)

    for _ in range(warmup):
        step_device()
    torch.cuda.synchronize()

    # device-resident timing with stage events
    ctx.reset_stage_times()
    ctx.set_profiling(True)
    launches0 = ctx.launches
    clocks = Clocks(local)
    barrier()
    torch.cuda.synchronize()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    for _ in range(steps):
        step_device()
    ev1.record(stream)
    torch.cuda.synchronize()
    barrier()
    clk = clocks.stop()
    ctx.set_profiling(False)
    launches = ctx.launches - launches0
    ms = ev0.elapsed_time(ev1)
    stages = ctx.stage_times()
    worst = max(c.residual_norm / c.rhs_norm for c in certs)

    # end-to-end through the host-buffer ABI
    ms_e2e = None
    if with_e2e:
        step_host()
        torch.cuda.synchronize()
        barrier()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(steps):
            step_host()
        e1.record(stream)
        torch.cuda.synchronize()
        barrier()
        ms_e2e = e0.elapsed_time(e1)
    ms, ms_e2e = reduce_max([ms, ms_e2e if ms_e2e is not None else 0.0])
    value = world * steps / (ms / 1e3)

    pk = peaks()
    nb = 128 if prec == t.MIXED else 64
    flops = lu_update_flops(n, nb) * steps
    gemm = stages.get("gemm", (0, 0.0))
    if prec == t.MIXED:
        # the update runs inside a seconds-long step: the sustained bf16 rate under the power cap
        bf16 = pk.get("bf16_tflops_sustained") or pk.get("bf16_tflops", 1590.0)
        tensor_peak = bf16 / 2.0  # TF32 dense = half of bf16 dense
        passes = 3.0 if os.environ.get("TCU_SPLIT") in ("tf32x3", "f16") else 2.0
        executed = passes * flops
        achieved = executed / (gemm[1] / 1e3) / 1e12 if gemm[1] else None
        roof = {"bound": "tensor", "achieved": achieved, "peak": tensor_peak, "unit": "TFLOP/s",
                "frac": achieved / tensor_peak if achieved else None,
                "traffic": TF32_TRAFFIC["ratio"] * update_launch_bytes(n, nb, os.environ.get("TCU_LU_PAIRS") != "0"),
                "traffic_note": TF32_TRAFFIC["note"],
                "kernel": f"tf32_update_kernel: split-TF32 tcgen05 trailing update ({passes:.0f} passes executed)",
                "useful_tflops": flops / (gemm[1] / 1e3) / 1e12 if gemm[1] else None,
                "peak_note": f"TF32 dense peak = half the sustained bf16 GEMM rate, {bf16} TFLOP/s "
                             f"(of measured: {pk.get('source')})"}
    else:
        achieved = flops / (gemm[1] / 1e3) / 1e12 if gemm[1] else None
        peak = fp64_peak if fp64_peak else 40.0
        roof = {"bound": "tensor", "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                "frac": achieved / peak if achieved else None, "traffic": None,
                "kernel": "zgemm_dmma_kernel: FP64 DMMA trailing update",
                "peak_note": "measured cuBLAS complex128 GEMM rate at 8192^2 (of measured)" if fp64_peak
                else "nominal FP64 tensor rate (no measurement in this run)"}
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": steps,
            "warmup": warmup, "ms_per_step": ms / steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "c64+c128 refine" if prec == t.MIXED else "c128", "data": "synthetic",
            "precision": precision, "parallelism": f"replicas x{world}", "config": workload_config(args.spheres),
            "max_rel_residual": worst, "roofline": roof,
            "stages_ms_per_step": {k: v[1] / steps for k, v in stages.items()},
            "gpu_launches": int(launches), "clocks": clk}
    if with_e2e:
        line["e2e"] = {"value": world * steps / (ms_e2e / 1e3), "unit": UNIT, "h2d_bytes_per_step": int(h2d),
                       "d2h_bytes_per_step": int(d2h)}
    X = X_d.cpu().numpy().reshape(n, p, order="F") if precision == args.precision else None
    return {"line": line, "X": X}


if __name__ == "__main__":
    main()
