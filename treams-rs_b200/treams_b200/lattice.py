"""2D Ewald lattice sums (treams_rs.lattice.lsumsw2d) and periodic arrays."""
from __future__ import annotations

import numpy as np

from ._lib import _check, _p, default_context, lib


def lsumsw2d_batch(lmax_sum: int, k, lattice, kpars, eta: float = 0.0, shift=None, ctx=None) -> np.ndarray:
    """D_lm(k, kpar, r) for every l <= lmax_sum (table index l*l+l+m) and every Bloch vector
    (nk, 2) (lattice.lsumsw2d, lattice::sum) at a shift r (default 0). A complex k with a
    positive imaginary part (a lossy embedding, Im k <= Re k / 2) takes the complex-wavenumber
    kernels; eta is a real split (0: automatic)."""
    ctx = ctx or default_context()
    a = np.ascontiguousarray(lattice, np.float64).reshape(2, 2)
    kp = np.ascontiguousarray(kpars, np.float64).reshape(-1, 2)
    out = np.zeros((kp.shape[0], (lmax_sum + 1) ** 2), np.complex128)
    kc = complex(k)
    if kc.imag != 0.0:
        kk = np.array([kc.real, kc.imag], np.float64)
        r = np.zeros(3) if shift is None else np.ascontiguousarray(shift, np.float64).reshape(3)
        _check(lib().tcu_lsumsw2d_complex_batch(ctx.handle, lmax_sum, _p(kk), _p(a), kp.shape[0], _p(kp), _p(r),
                                                float(eta), _p(out)))
    elif shift is None:
        _check(lib().tcu_lsumsw2d_batch(ctx.handle, lmax_sum, kc.real, _p(a), kp.shape[0], _p(kp), float(eta),
                                        _p(out)))
    else:
        r = np.ascontiguousarray(shift, np.float64).reshape(3)
        _check(lib().tcu_lsumsw2d_shift_batch(ctx.handle, lmax_sum, kc.real, _p(a), kp.shape[0], _p(kp), _p(r),
                                              float(eta), _p(out)))
    return out


def array_solve_batch(lmax: int, k0: float, radius: float, eps: complex, lattice, kpars, eta: float = 0.0,
                      ctx=None) -> np.ndarray:
    """X(kpar) = (I - T S(kpar))^-1 T for each Bloch vector: (nk, M, M)."""
    ctx = ctx or default_context()
    a = np.ascontiguousarray(lattice, np.float64).reshape(2, 2)
    kp = np.ascontiguousarray(kpars, np.float64).reshape(-1, 2)
    e = np.array([complex(eps)], np.complex128)
    M = 2 * lmax * (lmax + 2)
    out = np.empty((kp.shape[0], M, M), np.complex128)  # every entry is written by the library
    _check(lib().tcu_array_solve_batch(ctx.handle, lmax, float(k0), float(radius), _p(e), _p(a), kp.shape[0], _p(kp),
                                       float(eta), _p(out)))
    # the library writes each X column-major; the transposed view indexes X[k][row, col]
    return np.transpose(out, (0, 2, 1))
