"""CPU oracle — test infrastructure only.

ctypes binding of ``oracle/liboracle.so``, the C++ restatement of the treams-rs FP64
cluster path (``oracle.cpp``) and 2D Ewald lattice sums (``ewald.cpp``). Only the tests,
``__graft_entry__.smoke()`` and the CPU-baseline leg of ``bench.py`` import this module,
to check or time the CUDA library. The product never calls it.
"""
from __future__ import annotations

import ctypes
import pathlib
import subprocess

import numpy as np

HERE = pathlib.Path(__file__).resolve().parent
_LIB = None

c_int = ctypes.c_int
c_double = ctypes.c_double
P = ctypes.c_void_p


def build() -> None:
    subprocess.run(["make", "-s", "-C", str(HERE)], check=True)


def lib() -> ctypes.CDLL:
    global _LIB
    if _LIB is None:
        path = HERE / "liboracle.so"
        if not path.exists():
            build()
        _LIB = ctypes.CDLL(str(path))
        L = _LIB
        L.orc_wigner3j.restype = c_double
        L.orc_wigner3j.argtypes = [c_int] * 6
        L.orc_degrees.restype = c_int
        L.orc_degrees.argtypes = [c_int, c_int, c_int, c_int, c_int, P, c_int]
        L.orc_spherical_hankels.argtypes = [c_int, c_double, P]
        L.orc_spherical_j.argtypes = [c_int, c_double, c_double, P]
        L.orc_spherical_h.argtypes = [c_int, c_double, c_double, P]
        L.orc_solid_table.argtypes = [c_int, P, P]
        L.orc_plan_terms.restype = c_int
        L.orc_plan_terms.argtypes = [c_int]
        L.orc_translation_block.argtypes = [c_int, c_double, P, c_int, c_int, P]
        L.orc_mie_block.argtypes = [c_int, c_double, c_double, c_double, P]
        L.orc_cluster_operator.argtypes = [c_int, c_double, c_int, P, P, P, P, P]
        L.orc_plane_wave_expansion.argtypes = [c_int, c_int, P, c_int, P, P, P]
        L.orc_dense_solve.restype = c_int
        L.orc_dense_solve.argtypes = [c_int, c_int, P, P, P, c_int, P]
        L.orc_lu_solve.restype = c_int
        L.orc_lu_solve.argtypes = [c_int, P, P, c_int]
        L.orc_cross_sections.argtypes = [c_int, c_double, c_int, P, P, P, P, P]
        L.orc_iterative_apply.argtypes = [c_int, c_double, c_int, P, P, P, P, c_int, P]
        L.orc_iterative_solve.restype = c_int
        L.orc_iterative_solve.argtypes = [c_int, c_double, c_int, P, P, P, P, c_int, c_double, c_double,
                                          c_int, c_int, P, P, P]
        L.orc_gmres_dense.restype = c_int
        L.orc_gmres_dense.argtypes = [c_int, P, P, c_double, c_int, c_int, P, P, P]
        L.orc_upper_gamma.restype = c_int
        L.orc_upper_gamma.argtypes = [c_double, c_double, c_double, P]
        L.orc_kambe.restype = c_int
        L.orc_kambe.argtypes = [c_int, c_double, c_double, c_double, c_double, P]
        L.orc_lsumsw2d.restype = c_int
        L.orc_lsumsw2d.argtypes = [c_int, c_int, c_double, c_double, P, P, P, c_double, c_double, c_int, P]
        L.orc_lsumsw2d_table.restype = c_int
        L.orc_lsumsw2d_table.argtypes = [c_int, c_double, c_double, P, P, P, c_double, c_double, P]
        L.orc_array_solve.restype = c_int
        L.orc_array_solve.argtypes = [c_int, c_double, c_double, c_double, c_double, P, P, c_double, P]
    return _LIB


def _p(a: np.ndarray) -> int:
    return a.ctypes.data


def modes(lmax: int) -> list[tuple[int, int, int]]:
    return [(l, m, pol) for l in range(1, lmax + 1) for m in range(-l, l + 1) for pol in (1, 0)]


def wigner3j(j1, j2, j3, m1, m2, m3) -> float:
    return lib().orc_wigner3j(j1, j2, j3, m1, m2, m3)


def degrees(l, m, lam, mu, cross) -> list[int]:
    out = np.zeros(64, np.int32)
    k = lib().orc_degrees(l, m, lam, mu, int(cross), _p(out), 64)
    return [int(v) for v in out[:k]]


def spherical_hankels(last: int, x: float) -> np.ndarray:
    out = np.zeros(last + 1, np.complex128)
    lib().orc_spherical_hankels(last, float(x), _p(out))
    return out


def spherical_j(last: int, z: complex) -> np.ndarray:
    out = np.zeros(last + 1, np.complex128)
    lib().orc_spherical_j(last, z.real, z.imag, _p(out))
    return out


def spherical_h(last: int, z: complex) -> np.ndarray:
    out = np.zeros(last + 1, np.complex128)
    lib().orc_spherical_h(last, z.real, z.imag, _p(out))
    return out


def solid_table(order: int, unit) -> np.ndarray:
    u = np.ascontiguousarray(unit, np.float64)
    out = np.zeros((order + 1) ** 2, np.complex128)
    lib().orc_solid_table(order, _p(u), _p(out))
    return out


def plan_terms(lmax: int) -> int:
    return lib().orc_plan_terms(lmax)


def translation_block(lmax: int, k: float, disp, singular=True, helicity=True) -> np.ndarray:
    M = 2 * lmax * (lmax + 2)
    d = np.ascontiguousarray(disp, np.float64)
    out = np.zeros(M * M, np.complex128)
    lib().orc_translation_block(lmax, float(k), _p(d), int(singular), int(helicity), _p(out))
    return out.reshape(M, M).T.copy()  # column-major storage -> (row, col)


def mie_block(l: int, size: float, eps: complex) -> np.ndarray:
    out = np.zeros(4, np.complex128)
    lib().orc_mie_block(l, float(size), eps.real, eps.imag, _p(out))
    return out.reshape(2, 2)


def cluster_operator(lmax, k0, radii, eps, pos):
    """A = I - T C as an (n, n) array plus the T blocks (N, lmax, 2, 2)."""
    N = len(radii)
    M = 2 * lmax * (lmax + 2)
    n = N * M
    r = np.ascontiguousarray(radii, np.float64)
    e = np.ascontiguousarray(eps, np.complex128)
    x = np.ascontiguousarray(pos, np.float64)
    A = np.zeros((n, n), np.complex128, order="F")
    tb = np.zeros((N, lmax, 2, 2), np.complex128)
    lib().orc_cluster_operator(lmax, float(k0), N, _p(r), _p(e), _p(x), _p(A), _p(tb))
    return A, tb


def plane_wave_expansion(lmax, pos, kvecs, pols):
    N = len(pos)
    M = 2 * lmax * (lmax + 2)
    x = np.ascontiguousarray(pos, np.float64)
    kv = np.ascontiguousarray(kvecs, np.complex128)
    pl = np.ascontiguousarray(pols, np.int32)
    p = len(pl)
    out = np.zeros((N * M, p), np.complex128, order="F")
    lib().orc_plane_wave_expansion(lmax, N, _p(x), p, _p(kv), _p(pl), _p(out))
    return out


def dense_solve(lmax, A, tb, B):
    """Solve (I - T C) X = T B with the restated LU."""
    n, p = B.shape
    N = tb.shape[0]
    A = np.asfortranarray(A, np.complex128)
    tb = np.ascontiguousarray(tb, np.complex128)
    B = np.asfortranarray(B, np.complex128)
    X = np.zeros((n, p), np.complex128, order="F")
    st = lib().orc_dense_solve(lmax, N, _p(A), _p(tb), _p(B), p, _p(X))
    if st:
        raise RuntimeError(f"oracle dense solve failed with status {st}")
    return X


def lu_solve(A, B):
    A = np.asfortranarray(A, np.complex128)
    X = np.asfortranarray(B, np.complex128).copy(order="F")
    st = lib().orc_lu_solve(A.shape[0], _p(A), _p(X), X.shape[1] if X.ndim == 2 else 1)
    if st:
        raise RuntimeError(f"oracle LU failed with status {st}")
    return X


def cross_sections(lmax, k0, pos, x, b):
    xp = np.ascontiguousarray(pos, np.float64)
    xx = np.ascontiguousarray(x, np.complex128)
    bb = np.ascontiguousarray(b, np.complex128)
    sca = c_double()
    ext = c_double()
    lib().orc_cross_sections(lmax, float(k0), len(pos), _p(xp), _p(xx), _p(bb), ctypes.byref(sca), ctypes.byref(ext))
    return sca.value, ext.value


def iterative_apply(lmax, k0, radii, eps, pos, X):
    X = np.asfortranarray(X, np.complex128)
    if X.ndim == 1:
        X = X[:, None]
    r = np.ascontiguousarray(radii, np.float64)
    e = np.ascontiguousarray(eps, np.complex128)
    x = np.ascontiguousarray(pos, np.float64)
    Y = np.zeros_like(X, order="F")
    lib().orc_iterative_apply(lmax, float(k0), len(r), _p(r), _p(e), _p(x), _p(X), X.shape[1], _p(Y))
    return Y


def iterative_solve(lmax, k0, radii, eps, pos, B, rtol=1e-10, atol=0.0, restart=30, max_iterations=300):
    B = np.asfortranarray(B, np.complex128)
    if B.ndim == 1:
        B = B[:, None]
    p = B.shape[1]
    r = np.ascontiguousarray(radii, np.float64)
    e = np.ascontiguousarray(eps, np.complex128)
    x = np.ascontiguousarray(pos, np.float64)
    X = np.zeros_like(B, order="F")
    its = np.zeros(p, np.int32)
    res = np.zeros(p, np.float64)
    st = lib().orc_iterative_solve(lmax, float(k0), len(r), _p(r), _p(e), _p(x), _p(B), p, rtol, atol, restart,
                                   max_iterations, _p(X), _p(its), _p(res))
    return X, its, res, st


def gmres_dense(A, b, rtol=1e-10, restart=30, max_iterations=300):
    A = np.asfortranarray(A, np.complex128)
    b = np.ascontiguousarray(b, np.complex128)
    x = np.zeros_like(b)
    its = np.zeros(1, np.int32)
    res = np.zeros(1, np.float64)
    st = lib().orc_gmres_dense(A.shape[0], _p(A), _p(b), rtol, restart, max_iterations, _p(x), _p(its), _p(res))
    return x, int(its[0]), float(res[0]), st


def upper_gamma(a: float, z: complex) -> complex:
    """Gamma(a, z), principal branch; a zero imaginary part picks the side by its sign."""
    out = np.zeros(2)
    lib().orc_upper_gamma(float(a), z.real, z.imag, _p(out))
    return complex(out[0], out[1])


def kambe(n: int, z: complex, eta: complex) -> complex:
    out = np.zeros(2)
    lib().orc_kambe(int(n), z.real, z.imag, eta.real, eta.imag, _p(out))
    return complex(out[0], out[1])


_PARTS = {"full": 0, "real": 1, "reciprocal": 2}


def lsumsw2d(l: int, m: int, k: complex, lattice, kpar, r, eta: complex = 0.0, part: str = "full") -> complex:
    """One 2D spherical lattice sum D_lm (lattice/mod.rs:11-15) or one of its Ewald parts."""
    a = np.ascontiguousarray(lattice, np.float64).reshape(4)
    kp = np.ascontiguousarray(kpar, np.float64).reshape(2)
    rr = np.ascontiguousarray(r, np.float64).reshape(3)
    out = np.zeros(2)
    k, eta = complex(k), complex(eta)
    st = lib().orc_lsumsw2d(l, m, k.real, k.imag, _p(a), _p(kp), _p(rr), eta.real, eta.imag, _PARTS[part], _p(out))
    if st:
        raise ValueError(f"oracle lattice sum failed with status {st}")
    return complex(out[0], out[1])


def lsumsw2d_table(lmax: int, k: complex, lattice, kpar, r=(0.0, 0.0, 0.0), eta: complex = 0.0) -> np.ndarray:
    """Every D_lm with l <= lmax, table index l*l+l+m."""
    a = np.ascontiguousarray(lattice, np.float64).reshape(4)
    kp = np.ascontiguousarray(kpar, np.float64).reshape(2)
    rr = np.ascontiguousarray(r, np.float64).reshape(3)
    out = np.zeros((lmax + 1) ** 2, np.complex128)
    k, eta = complex(k), complex(eta)
    st = lib().orc_lsumsw2d_table(lmax, k.real, k.imag, _p(a), _p(kp), _p(rr), eta.real, eta.imag, _p(out))
    if st:
        raise ValueError(f"oracle lattice sum failed with status {st}")
    return out


def array_solve(lmax: int, k0: float, radius: float, eps: complex, lattice, kpar, eta: float = 0.0) -> np.ndarray:
    """X = (I - T S(kpar))^-1 T of a periodic array of one sphere per cell, (M, M)."""
    a = np.ascontiguousarray(lattice, np.float64).reshape(4)
    kp = np.ascontiguousarray(kpar, np.float64).reshape(2)
    M = 2 * lmax * (lmax + 2)
    out = np.zeros(M * M, np.complex128)
    eps = complex(eps)
    st = lib().orc_array_solve(lmax, k0, radius, eps.real, eps.imag, _p(a), _p(kp), float(eta), _p(out))
    if st:
        raise ValueError(f"oracle array solve failed with status {st}")
    return out.reshape(M, M, order="F")



def apply_t(lmax, tb, B):
    """T B for the per-sphere 2x2 Mie blocks tb (N, lmax, 2, 2) in mode order."""
    N = tb.shape[0]
    M = 2 * lmax * (lmax + 2)
    B = np.asarray(B, np.complex128)
    squeeze = B.ndim == 1
    if squeeze:
        B = B[:, None]
    degrees = np.array([l for l in range(1, lmax + 1) for _ in range(2 * l + 1)])
    Tq = tb[:, degrees - 1]                                  # (N, M/2, 2, 2)
    Bq = B.reshape(N, M // 2, 2, B.shape[1])
    out = np.einsum("nqab,nqbp->nqap", Tq, Bq).reshape(N * M, B.shape[1])
    return out[:, 0] if squeeze else np.asfortranarray(out)


def lapack_cluster_solve(lmax, k0, radii, eps, pos, B):
    """X = (I - T C)^-1 T B with the oracle's FP64 assembly and LAPACK zgetrf/zgetrs
    (scipy, all host threads), factoring in place so the host holds one n x n copy."""
    import scipy.linalg

    A, tb = cluster_operator(lmax, k0, radii, eps, pos)
    TB = apply_t(lmax, tb, B)
    lu, piv = scipy.linalg.lu_factor(A, overwrite_a=True, check_finite=False)
    del A
    return scipy.linalg.lu_solve((lu, piv), TB, check_finite=False)


# ---- learned preconditioner: restatement of the graph network and its training loss ----------
GNN_H, GNN_NF, GNN_EF = 16, 6, 5


def gnn_layout(lmax):
    """Offsets of the weight vector: W1 (16x6), b1, W2 (16x37), b2, W3 (16x37), b3, W4 (2L^2 x 16), b4."""
    H, nin, no = GNN_H, 2 * GNN_H + GNN_EF, 2 * lmax * lmax
    sizes = [("W1", (H, GNN_NF)), ("b1", (H,)), ("W2", (H, nin)), ("b2", (H,)), ("W3", (H, nin)), ("b3", (H,)),
             ("W4", (no, H)), ("b4", (no,))]
    out, o = {}, 0
    for name, shape in sizes:
        size = int(np.prod(shape))
        out[name] = (o, shape)
        o += size
    return out, o


def gnn_graph(k0, radii, eps, pos, reach_diameters=3.0):
    """Neighbours closer than reach_diameters * 2 max(radius) (rows sorted), node features
    [deg/12, sum 1/(kd)/8, sum 1/(kd)^3/4, |r - centroid|/max|r - centroid|, k r, Re eps/8] and
    edge features [1/(kd), 1/(kd)^2, 1/(kd)^3, kd/4, d/cutoff]."""
    pos = np.asarray(pos, float)
    N = len(pos)
    cutoff = 2.0 * reach_diameters * float(np.max(radii))
    D = np.linalg.norm(pos[:, None] - pos[None], axis=2)
    rows, nbrs = [], []
    for i in range(N):
        for j in range(N):
            if j != i and D[i, j] <= cutoff:
                rows.append(i)
                nbrs.append(j)
    rows, nbrs = np.array(rows, int), np.array(nbrs, int)
    d = D[rows, nbrs]
    kd = k0 * d
    E = np.stack([1 / kd, 1 / kd**2, 1 / kd**3, kd / 4, d / cutoff], axis=1) if len(d) else np.zeros((0, 5))
    c = pos.mean(axis=0)
    rc = np.linalg.norm(pos - c, axis=1)
    R = rc.max() if rc.max() > 0 else 1.0
    X = np.zeros((N, GNN_NF))
    for i in range(N):
        sel = rows == i
        X[i] = [sel.sum() / 12, np.sum(1 / kd[sel]) / 8, np.sum(1 / kd[sel] ** 3) / 4, rc[i] / R, k0 * radii[i],
                np.real(eps[i]) / 8]
    return rows, nbrs, X, E


def gnn_theta(lmax, weights, rows, nbrs, X, E):
    """Raw network outputs per edge (nnz, 2 lmax^2): Theta = 1 + out[2q] + i out[2q+1]."""
    lay, total = gnn_layout(lmax)
    w = np.asarray(weights, float)
    assert w.size == total
    get = lambda name: w[lay[name][0]:lay[name][0] + int(np.prod(lay[name][1]))].reshape(lay[name][1])  # noqa: E731
    h = np.tanh(X @ get("W1").T + get("b1"))
    N = X.shape[0]
    g = h.copy()
    for i in range(N):
        sel = np.where(rows == i)[0]
        if len(sel):
            z = np.concatenate([np.repeat(h[i:i + 1], len(sel), 0), h[nbrs[sel]], E[sel]], axis=1)
            g[i] = h[i] + np.tanh(z @ get("W2").T + get("b2")).mean(axis=0)
    z = np.concatenate([g[rows], g[nbrs], E], axis=1)
    a = np.tanh(z @ get("W3").T + get("b3"))
    return a @ get("W4").T + get("b4")


def gnn_near_apply(lmax, k0, pos, tb, rows, nbrs, theta, R):
    """M R = R + T sum_j (Theta_ij o C_ij) R_j over the near-field edges."""
    M = 2 * lmax * (lmax + 2)
    nlm = M // 2
    deg = np.array([l for l in range(1, lmax + 1) for _ in range(2 * l + 1)])
    Y = np.array(R, complex, copy=True)
    CR = np.zeros_like(Y)
    for e, (i, j) in enumerate(zip(rows, nbrs)):
        blk = translation_block(lmax, k0, np.asarray(pos[i]) - np.asarray(pos[j]), singular=True, helicity=True)
        th = 1.0 + theta[e, 0::2] + 1j * theta[e, 1::2]          # (lmax^2,), index (lam-1) L + (l-1)
        scale = th[(deg[:, None] - 1) * lmax + (deg[None, :] - 1)]  # (nlm dest, nlm src)
        S = np.repeat(np.repeat(scale, 2, axis=0), 2, axis=1)
        CR[i * M:(i + 1) * M] += (blk * S) @ R[j * M:(j + 1) * M]
    Y += apply_t(lmax, tb, CR)
    return Y


def gnn_loss(lmax, k0, radii, eps, pos, R, weights, reach_diameters=3.0, A=None, tb=None):
    """sum_p ||r_p - A M_Theta r_p||^2 with the dense oracle operator A = I - T C."""
    if A is None:
        A, tb = cluster_operator(lmax, k0, radii, eps, pos)
    rows, nbrs, X, E = gnn_graph(k0, np.asarray(radii), np.asarray(eps), pos, reach_diameters)
    theta = gnn_theta(lmax, weights, rows, nbrs, X, E)
    Y = gnn_near_apply(lmax, k0, np.asarray(pos), tb, rows, nbrs, theta, np.asarray(R).reshape(A.shape[0], -1))
    Rr = np.asarray(R).reshape(A.shape[0], -1)
    return float(np.sum(np.abs(Rr - A @ Y) ** 2))
