"""ctypes binding of include/treams_cuda.h (libtreams_b200.so)."""
from __future__ import annotations

import ctypes
import pathlib
import threading
import weakref
from dataclasses import dataclass

import numpy as np

PKG_ROOT = pathlib.Path(__file__).resolve().parent.parent
_LIB_PATH = PKG_ROOT / "libtreams_b200.so"

FP64 = 0
MIXED = 1
PRECOND = {"none": 0, "block_jacobi": 1, "learned": 2, "two_level": 3}

c_int, c_double, c_size, P = ctypes.c_int, ctypes.c_double, ctypes.c_size_t, ctypes.c_void_p


class TreamsCudaError(RuntimeError):
    """A device failure or a timed-out device-side wait."""


class Certificate(ctypes.Structure):
    _fields_ = [("iterations", c_int), ("residual_norm", c_double), ("rhs_norm", c_double)]

    def __repr__(self) -> str:
        return (f"Certificate(iterations={self.iterations}, residual_norm={self.residual_norm:.3e}, "
                f"rhs_norm={self.rhs_norm:.3e})")


class GmresOptions(ctypes.Structure):
    _fields_ = [("rtol", c_double), ("atol", c_double), ("restart", c_int), ("max_iterations", c_int)]


SIGNATURES = {
    "tcu_context_create": (c_int, [c_int, ctypes.POINTER(P)]),
    "tcu_context_destroy": (c_int, [P]),
    "tcu_context_stream": (P, [P]),
    "tcu_last_error_message": (ctypes.c_char_p, []),
    "tcu_context_launches": (ctypes.c_longlong, [P]),
    "tcu_context_fallbacks": (ctypes.c_longlong, [P]),
    "tcu_context_set_refinement": (c_int, [P, c_double, c_double]),
    "tcu_context_wait_selftest": (c_int, [P, c_double]),
    "tcu_context_autotune": (c_int, [P, ctypes.POINTER(c_size), c_int, P, P, P]),
    "tcu_context_set_profiling": (c_int, [P, c_int]),
    "tcu_context_stage_time": (c_int, [P, c_int, ctypes.POINTER(ctypes.c_longlong), ctypes.POINTER(c_double)]),
    "tcu_context_reset_stage_times": (c_int, [P]),
    "tcu_translation_block": (c_int, [P, c_int, c_double, P, c_int, c_int, P]),
    "tcu_translate": (c_int, [P, c_size, P, P, c_int, c_int, P]),
    "tcu_wigner3j": (c_double, [c_int] * 6),
    "tcu_mie_blocks": (c_int, [P, c_int, c_double, c_size, P, P, P]),
    "tcu_plane_wave_expansion": (c_int, [P, c_int, c_size, P, c_int, P, P, P]),
    "tcu_cross_sections": (c_int, [P, c_int, c_double, c_size, P, c_int, P, P, P, P]),
    "tcu_sphere_cluster_factor": (c_int, [P, c_int, c_double, c_size, P, P, P, c_int, ctypes.POINTER(P)]),
    "tcu_sphere_cluster_factor_dev": (c_int, [P, c_int, c_double, c_size, P, P, P, c_int, ctypes.POINTER(P)]),
    "tcu_factor_solve": (c_int, [P, P, c_int, P, P]),
    "tcu_factor_solve_dev": (c_int, [P, P, c_int, P, P]),
    "tcu_factor_dimension": (c_size, [P]),
    "tcu_factor_solve_adjoint": (c_int, [P, P, c_int, P, P]),
    "tcu_factor_interacting_tmatrix": (c_int, [P, P]),
    "tcu_factor_global_tmatrix": (c_int, [P, c_int, P, P]),
    "tcu_factor_pullback_incident": (c_int, [P, P, c_int, P, P]),
    "tcu_iterative_pullback_incident": (c_int, [P, c_int, c_double, c_size, P, P, P, P, c_int, P, P, P]),
    "tcu_factor_destroy": (c_int, [P]),
    "tcu_cluster_operator": (c_int, [P, c_int, c_double, c_size, P, P, P, P]),
    "tcu_cluster_apply": (c_int, [P, c_int, c_double, c_size, P, P, P, c_int, P, P]),
    "tcu_cluster_apply_noalloc": (c_int, [P, c_int, c_double, c_size, P, P, P, c_int, P, P]),
    "tcu_iterative_solve": (c_int, [P, c_int, c_double, c_size, P, P, P, P, c_int, P, c_int, P, P]),
    "tcu_batch_solve": (c_int, [P, c_size, P, c_int, P]),
    "tcu_context_set_learned_weights": (c_int, [P, c_double, c_size, P]),
    "tcu_learned_weight_count": (c_size, [c_int]),
    "tcu_learned_problem_create": (c_int, [P, c_int, c_double, c_size, P, P, P, c_int, P, ctypes.POINTER(P)]),
    "tcu_learned_problem_loss_grad": (c_int, [P, P, P, P]),
    "tcu_learned_problem_probes": (c_int, [P, P]),
    "tcu_learned_problem_destroy": (c_int, [P]),
    "tcu_lsumsw2d_batch": (c_int, [P, c_int, c_double, P, c_size, P, c_double, P]),
    "tcu_lsumsw2d_shift_batch": (c_int, [P, c_int, c_double, P, c_size, P, P, c_double, P]),
    "tcu_lsumsw2d_complex_batch": (c_int, [P, c_int, P, P, c_size, P, P, c_double, P]),
    "tcu_array_solve_batch": (c_int, [P, c_int, c_double, c_double, P, P, c_size, P, c_double, P]),
}

_lib = None
_lock = threading.Lock()


def library_path() -> pathlib.Path:
    return _LIB_PATH


def lib() -> ctypes.CDLL:
    global _lib
    with _lock:
        if _lib is None:
            if not _LIB_PATH.exists():
                raise ImportError(
                    f"{_LIB_PATH} is missing: build it with `make -C treams-rs_b200` (there is no CPU fallback)")
            handle = ctypes.CDLL(str(_LIB_PATH))
            for name, (res, args) in SIGNATURES.items():
                fn = getattr(handle, name)
                fn.restype = res
                fn.argtypes = args
            _lib = handle
    return _lib


def _check(status: int) -> None:
    if status == 0:
        return
    msg = lib().tcu_last_error_message().decode()
    if status == 6:
        raise MemoryError(msg)
    if status in (7, 8):
        raise TreamsCudaError(msg)
    raise ValueError(msg)  # InvalidInput, SpecialFunction, NonFinite, NotConverged, Singular


def _p(a: np.ndarray) -> int:
    return a.ctypes.data


class Context:
    """One CUDA stream and its workspaces on one device (tcu_context)."""

    def __init__(self, device: int = 0):
        h = P()
        _check(lib().tcu_context_create(device, ctypes.byref(h)))
        self.handle = h
        self._factors = weakref.WeakSet()  # closed before the context

    @property
    def stream(self) -> int:
        return lib().tcu_context_stream(self.handle)

    @property
    def launches(self) -> int:
        return lib().tcu_context_launches(self.handle)

    STAGES = ("assemble", "panel", "swap", "trsm", "gemm", "pack", "solve", "apply", "mie", "lattice", "small_lu",
              "coarse", "near")

    def set_refinement(self, target: float = 1e-13, fallback_above: float = 1e-12) -> None:
        """Refinement stop tolerance and the residual above which mixed solves finish in FP64."""
        _check(lib().tcu_context_set_refinement(self.handle, float(target), float(fallback_above)))

    def wait_selftest(self, limit: float = 0.05) -> None:
        """Run the LU panel's grid barrier with one arrival missing; its bounded wait gives up
        after `limit` seconds and this raises TreamsCudaError (status TCU_TIMEOUT), leaving the
        context usable."""
        _check(lib().tcu_context_wait_selftest(self.handle, float(limit)))

    def autotune(self) -> dict:
        """Measure the FP64/mixed crossover of batched solves (tcu_context_autotune): returns
        {"crossover": unknowns, "sizes": [...], "ms_fp64": [...], "ms_mixed": [...]}."""
        cross = c_size()
        sizes = np.zeros(6, np.uint64)
        f64 = np.zeros(6)
        mix = np.zeros(6)
        _check(lib().tcu_context_autotune(self.handle, ctypes.byref(cross), 6, _p(sizes), _p(f64), _p(mix)))
        return {"crossover": int(cross.value), "sizes": [int(v) for v in sizes], "ms_fp64": f64.tolist(),
                "ms_mixed": mix.tolist()}

    @property
    def fallbacks(self) -> int:
        """Mixed solves finished by an FP64 factor (refinement stalled)."""
        return lib().tcu_context_fallbacks(self.handle)

    def set_learned_weights(self, weights=None, reach: float = 0.0) -> None:
        """Network weights (None: the compiled-in ones) and near-field reach in sphere diameters
        (<= 0: the compiled-in 3) of the learned and two-level preconditioners."""
        w = np.zeros(0) if weights is None else np.ascontiguousarray(weights, np.float64)
        _check(lib().tcu_context_set_learned_weights(self.handle, float(reach), w.size, _p(w) if w.size else None))

    def set_profiling(self, on: bool) -> None:
        _check(lib().tcu_context_set_profiling(self.handle, int(on)))

    def reset_stage_times(self) -> None:
        _check(lib().tcu_context_reset_stage_times(self.handle))

    def stage_times(self) -> dict:
        """{stage: (launches, total_ms)} from CUDA events on the context stream."""
        out = {}
        for i, name in enumerate(self.STAGES):
            n = ctypes.c_longlong()
            ms = c_double()
            _check(lib().tcu_context_stage_time(self.handle, i, ctypes.byref(n), ctypes.byref(ms)))
            if n.value:
                out[name] = (n.value, ms.value)
        return out

    def close(self) -> None:
        if self.handle:
            for f in list(self._factors):
                f.close()
            lib().tcu_context_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


_default = None


def default_context() -> Context:
    global _default
    if _default is None:
        _default = Context(0)
    return _default


def _geom(radii, eps, positions):
    r = np.ascontiguousarray(radii, np.float64).reshape(-1)
    e = np.ascontiguousarray(np.broadcast_to(np.asarray(eps, np.complex128), r.shape))
    x = np.ascontiguousarray(positions, np.float64).reshape(-1, 3)
    if x.shape[0] != r.shape[0]:
        raise ValueError("require one position per sphere")
    return r, e, x


def modes(lmax: int) -> list[tuple[int, int, int]]:
    """Mode order of one sphere (sw/mod.rs:114-125): l, m = -l..l, pol 1 then pol 0."""
    return [(l, m, pol) for l in range(1, lmax + 1) for m in range(-l, l + 1) for pol in (1, 0)]


def translation_block(lmax: int, k: float, displacement, singular: bool = True, helicity: bool = True,
                      ctx: Context | None = None) -> np.ndarray:
    """(M, M) translation block from a source to a destination at displacement
    destination - source (TranslationPlan::evaluate, sw/plan.rs:282)."""
    ctx = ctx or default_context()
    M = 2 * lmax * (lmax + 2)
    d = np.ascontiguousarray(displacement, np.float64)
    out = np.zeros(M * M, np.complex128)
    _check(lib().tcu_translation_block(ctx.handle, lmax, float(k), _p(d), int(singular), int(helicity), _p(out)))
    return out.reshape(M, M).T.copy()


def mie_blocks(lmax: int, k0: float, radii, eps, ctx: Context | None = None) -> np.ndarray:
    """(N, lmax, 2, 2) Mie blocks in mode order (tmatrix::sphere, coeffs::mie)."""
    ctx = ctx or default_context()
    r = np.ascontiguousarray(radii, np.float64).reshape(-1)
    e = np.ascontiguousarray(np.broadcast_to(np.asarray(eps, np.complex128), r.shape))
    out = np.zeros((r.size, lmax, 2, 2), np.complex128)
    _check(lib().tcu_mie_blocks(ctx.handle, lmax, float(k0), r.size, _p(r), _p(e), _p(out)))
    return out


def plane_wave_expansion(lmax: int, positions, kvecs, pols, ctx: Context | None = None) -> np.ndarray:
    """(n, p) regular expansion of plane waves (pw::expansion, pw/expand.rs:308)."""
    ctx = ctx or default_context()
    x = np.ascontiguousarray(positions, np.float64).reshape(-1, 3)
    kv = np.ascontiguousarray(kvecs, np.complex128).reshape(-1, 3)
    pl = np.ascontiguousarray(pols, np.int32).reshape(-1)
    n = x.shape[0] * 2 * lmax * (lmax + 2)
    out = np.zeros((n, pl.size), np.complex128, order="F")
    _check(lib().tcu_plane_wave_expansion(ctx.handle, lmax, x.shape[0], _p(x), pl.size, _p(kv), _p(pl), _p(out)))
    return out


def cross_sections(lmax: int, k0: float, positions, scattered, incident, ctx: Context | None = None):
    """(sca, ext) per column, as TMatrix._cross_sections with flux 0.5 (_tmatrix.py:413)."""
    ctx = ctx or default_context()
    x = np.ascontiguousarray(positions, np.float64).reshape(-1, 3)
    xs = np.asfortranarray(scattered, np.complex128)
    bs = np.asfortranarray(incident, np.complex128)
    if xs.ndim == 1:
        xs, bs = xs[:, None], bs[:, None]
    p = xs.shape[1]
    sca = np.zeros(p)
    ext = np.zeros(p)
    _check(lib().tcu_cross_sections(ctx.handle, lmax, float(k0), x.shape[0], _p(x), p, _p(xs), _p(bs), _p(sca),
                                    _p(ext)))
    return sca, ext


def cluster_operator(lmax, k0, radii, eps, positions, ctx: Context | None = None) -> np.ndarray:
    """The dense operator I - T C, complex128 (n, n)."""
    ctx = ctx or default_context()
    r, e, x = _geom(radii, eps, positions)
    n = r.size * 2 * lmax * (lmax + 2)
    out = np.zeros((n, n), np.complex128, order="F")
    _check(lib().tcu_cluster_operator(ctx.handle, lmax, float(k0), r.size, _p(r), _p(e), _p(x), _p(out)))
    return out


def cluster_apply(lmax, k0, radii, eps, positions, vectors, ctx: Context | None = None) -> np.ndarray:
    """(I - T C) x without forming C (IterativeSphereCluster::apply)."""
    ctx = ctx or default_context()
    r, e, x = _geom(radii, eps, positions)
    v = np.asfortranarray(vectors, np.complex128)
    squeeze = v.ndim == 1
    if squeeze:
        v = v[:, None]
    out = np.zeros_like(v, order="F")
    _check(lib().tcu_cluster_apply(ctx.handle, lmax, float(k0), r.size, _p(r), _p(e), _p(x), v.shape[1], _p(v),
                                   _p(out)))
    return out[:, 0] if squeeze else out


class InteractionFactor:
    """LU factor of I - T C on the device (InteractionFactor, cluster/interaction.rs:181)."""

    def __init__(self, handle, ctx: Context, precision: int):
        self.handle = handle
        self.ctx = ctx
        self.precision = precision
        ctx._factors.add(self)
        self.dimension = int(lib().tcu_factor_dimension(handle))

    def solve(self, incident) -> tuple[np.ndarray, list[Certificate]]:
        """Solve (I - T C) X = T B for the supplied columns (InteractionFactor::solve)."""
        b = np.asfortranarray(incident, np.complex128)
        squeeze = b.ndim == 1
        if squeeze:
            b = b[:, None]
        if b.shape[0] != self.dimension or b.shape[1] == 0:
            raise ValueError("require finite channel-by-illumination columns matching the factorization")
        x = np.zeros_like(b, order="F")
        certs = (Certificate * b.shape[1])()
        _check(lib().tcu_factor_solve(self.handle, _p(b), b.shape[1], _p(x), certs))
        return (x[:, 0] if squeeze else x), list(certs)

    def _adjoint(self, cotangent, fn):
        g = np.asfortranarray(cotangent, np.complex128)
        squeeze = g.ndim == 1
        if squeeze:
            g = g[:, None]
        if g.shape[0] != self.dimension or g.shape[1] == 0:
            raise ValueError("require finite channel-by-illumination columns matching the factorization")
        out = np.zeros_like(g, order="F")
        certs = (Certificate * g.shape[1])()
        _check(fn(self.handle, _p(g), g.shape[1], _p(out), certs))
        return (out[:, 0] if squeeze else out), list(certs)

    def interacting_tmatrix(self) -> np.ndarray:
        """X = (I - T C)^-1 T, (n, n) (cluster::interaction, cluster/interaction.rs:292)."""
        X = np.zeros((self.dimension, self.dimension), np.complex128, order="F")
        _check(lib().tcu_factor_interacting_tmatrix(self.handle, _p(X)))
        return X

    def global_tmatrix(self, lmax_global: int, origin=(0.0, 0.0, 0.0)) -> np.ndarray:
        """The cluster's T-matrix in one spherical basis of degree lmax_global at origin
        (the expand of a cluster T-matrix into SphericalBasis.default(lmax_global))."""
        o = np.ascontiguousarray(origin, np.float64)
        Mg = 2 * lmax_global * (lmax_global + 2)
        out = np.zeros((Mg, Mg), np.complex128, order="F")
        _check(lib().tcu_factor_global_tmatrix(self.handle, int(lmax_global), _p(o), _p(out)))
        return out

    def solve_adjoint(self, cotangent):
        """Y = (I - T C)^-H G with the saved factor (Lu::solve_adjoint_in_place)."""
        return self._adjoint(cotangent, lib().tcu_factor_solve_adjoint)

    def pullback_incident(self, cotangent):
        """Gradient of the incident columns: T^H (I - T C)^-H G
        (InteractionFactor::pullback_incident, cluster/interaction.rs:221)."""
        return self._adjoint(cotangent, lib().tcu_factor_pullback_incident)

    def close(self) -> None:
        if self.handle:
            if self.ctx.handle:
                lib().tcu_factor_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def sphere_cluster_factor(lmax: int, k0: float, radii, eps, positions, precision: str | int = "fp64",
                          ctx: Context | None = None) -> InteractionFactor:
    """Assemble and factor I - T C (cluster::sphere_cluster_factor, cluster/spheres.rs:85).

    precision "fp64" is the plain drop-in; "mixed" factors in complex64 with split-TF32
    tensor-core updates and refines every solve in FP64."""
    ctx = ctx or default_context()
    prec = {"fp64": FP64, "mixed": MIXED}.get(precision, precision)
    r, e, x = _geom(radii, eps, positions)
    h = P()
    _check(lib().tcu_sphere_cluster_factor(ctx.handle, lmax, float(k0), r.size, _p(r), _p(e), _p(x), int(prec),
                                           ctypes.byref(h)))
    return InteractionFactor(h, ctx, int(prec))


@dataclass
class IterativeSolution:
    value: np.ndarray
    convergence: list


def learned_weight_count(lmax: int) -> int:
    return int(lib().tcu_learned_weight_count(lmax))


class LearnedProblem:
    """One training cluster of the learned preconditioner's graph network on the GPU
    (tcu_learned_problem): loss_grad(weights) -> (loss, gradient) from the device's forward and
    backward kernels; probes() -> the coarse-corrected unit-norm probe vectors (n, nprobe)."""

    def __init__(self, lmax, k0, radii, eps, positions, V, ctx: Context | None = None):
        self.ctx = ctx or default_context()
        r, e, x = _geom(radii, eps, positions)
        V = np.asfortranarray(V, np.complex128)
        if V.ndim == 1:
            V = V[:, None]
        self.lmax, self.n, self.nprobe = lmax, V.shape[0], V.shape[1]
        self.nweights = learned_weight_count(lmax)
        h = P()
        _check(lib().tcu_learned_problem_create(self.ctx.handle, lmax, float(k0), r.size, _p(r), _p(e), _p(x),
                                                V.shape[1], _p(V), ctypes.byref(h)))
        self.handle = h

    def loss_grad(self, weights):
        w = np.ascontiguousarray(weights, np.float64)
        if w.size != self.nweights:
            raise ValueError(f"expected {self.nweights} weights")
        loss = c_double()
        grad = np.zeros(self.nweights)
        _check(lib().tcu_learned_problem_loss_grad(self.handle, _p(w), ctypes.byref(loss), _p(grad)))
        return loss.value, grad

    def probes(self) -> np.ndarray:
        out = np.zeros((self.n, self.nprobe), np.complex128, order="F")
        _check(lib().tcu_learned_problem_probes(self.handle, _p(out)))
        return out

    def close(self) -> None:
        if self.handle:
            lib().tcu_learned_problem_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class ClusterDesc(ctypes.Structure):
    _fields_ = [("lmax", c_int), ("k0", c_double), ("N", c_size), ("radii", P), ("eps", P), ("positions", P),
                ("B", P), ("p", c_int), ("X", P), ("certificates", P)]


PRECISION = {"fp64": 0, "mixed": 1, "auto": 2}


def batch_solve(clusters, precision: str = "auto", ctx: Context | None = None):
    """Solve independent clusters in one call (tcu_batch_solve): clusters is a list of
    (lmax, k0, radii, eps, positions, B) with B (n, p); returns (list of X, list of certificate
    lists, processing order). Largest clusters first; one operator resident at a time."""
    ctx = ctx or default_context()
    keep, descs, outs, certs = [], [], [], []
    for lmax, k0, radii, eps, positions, B in clusters:
        r, e, x = _geom(radii, eps, positions)
        b = np.asfortranarray(B, np.complex128)
        if b.ndim == 1:
            b = b[:, None]
        X = np.zeros_like(b, order="F")
        cs = (Certificate * b.shape[1])()
        keep += [r, e, x, b]
        outs.append(X)
        certs.append(cs)
        descs.append(ClusterDesc(lmax, float(k0), r.size, _p(r), _p(e), _p(x), _p(b), b.shape[1], _p(X),
                                 ctypes.addressof(cs)))
    arr = (ClusterDesc * len(descs))(*descs)
    order = (c_int * max(1, len(descs)))()
    _check(lib().tcu_batch_solve(ctx.handle, len(descs), arr, PRECISION[precision], order))
    return outs, [list(c) for c in certs], list(order)[:len(descs)]


class SphereCluster:
    """Matrix-free cluster solved by GMRES (IterativeSphereCluster, cluster/iterative.rs:39;
    python/treams_rs/iterative.py defaults rtol 1e-10, restart 30, max 300)."""

    def __init__(self, lmax: int, k0: float, radii, eps, positions, ctx: Context | None = None):
        self.ctx = ctx or default_context()
        self.lmax, self.k0 = lmax, float(k0)
        self.radii, self.eps, self.positions = _geom(radii, eps, positions)
        self.dimension = self.radii.size * 2 * lmax * (lmax + 2)

    def apply(self, vectors) -> np.ndarray:
        return cluster_apply(self.lmax, self.k0, self.radii, self.eps, self.positions, vectors, self.ctx)

    def solve(self, incident, rtol: float = 1e-10, atol: float = 0.0, restart: int = 30, max_iterations: int = 300,
              preconditioner: str = "none") -> IterativeSolution:
        b = np.asfortranarray(incident, np.complex128)
        squeeze = b.ndim == 1
        if squeeze:
            b = b[:, None]
        x = np.zeros_like(b, order="F")
        certs = (Certificate * b.shape[1])()
        opt = GmresOptions(rtol, atol, restart, max_iterations)
        _check(lib().tcu_iterative_solve(self.ctx.handle, self.lmax, self.k0, self.radii.size, _p(self.radii),
                                         _p(self.eps), _p(self.positions), _p(b), b.shape[1], ctypes.byref(opt),
                                         PRECOND[preconditioner], _p(x), certs))
        return IterativeSolution(x[:, 0] if squeeze else x, list(certs))

    def pullback_incident(self, cotangent, rtol: float = 1e-10, atol: float = 0.0, restart: int = 30,
                          max_iterations: int = 300) -> IterativeSolution:
        """Incident-field gradient T^H (I - T C)^-H G by adjoint GMRES (the `incident` part of
        IterativeSphereCluster::pullback, cluster/iterative.rs:460)."""
        g = np.asfortranarray(cotangent, np.complex128)
        squeeze = g.ndim == 1
        if squeeze:
            g = g[:, None]
        out = np.zeros_like(g, order="F")
        certs = (Certificate * g.shape[1])()
        opt = GmresOptions(rtol, atol, restart, max_iterations)
        _check(lib().tcu_iterative_pullback_incident(self.ctx.handle, self.lmax, self.k0, self.radii.size,
                                                     _p(self.radii), _p(self.eps), _p(self.positions), _p(g),
                                                     g.shape[1], ctypes.byref(opt), _p(out), certs))
        return IterativeSolution(out[:, 0] if squeeze else out, list(certs))
