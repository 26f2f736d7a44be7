"""Spherical-wave translations (treams_rs.sw): per-entry coefficients and whole blocks."""
from __future__ import annotations

import numpy as np

from ._lib import _check, _p, default_context, lib, modes, translation_block  # noqa: F401


def translate(lambda_, mu, pol, l, m, qol, kr, theta, phi, poltype: str | None = None, singular: bool = True,
              ctx=None):
    """Translation coefficient of mode pairs (sw.translate, python/treams_rs/sw.py:70).

    Destination mode (lambda_, mu, pol), source mode (l, m, qol); kr, theta, phi are the
    spherical coordinates of k (r_destination - r_source), real or complex. Helicity modes
    (the default) give A + (2 pol - 1) B for equal helicities and 0 otherwise; parity modes
    A for equal and B for different parities. The arguments broadcast like a ufunc; the
    result is complex128 of the broadcast shape (a Python complex for scalars)."""
    ctx = ctx or default_context()
    helicity = poltype in (None, "helicity")
    if not helicity and poltype != "parity":
        raise ValueError(f"unknown polarization type {poltype!r}")
    arrays = np.broadcast_arrays(*(np.asarray(v) for v in (lambda_, mu, pol, l, m, qol, kr, theta, phi)))
    shape = arrays[0].shape
    labels = np.ascontiguousarray(np.stack([a.reshape(-1) for a in arrays[:6]], axis=1), np.int32)
    if not all(np.array_equal(np.asarray(a).astype(np.int64), np.asarray(a)) for a in arrays[:6]):
        raise ValueError("mode labels must be integers")
    args = np.ascontiguousarray(np.stack([np.asarray(a, np.complex128).reshape(-1) for a in arrays[6:]], axis=1))
    count = labels.shape[0]
    out = np.zeros(count, np.complex128)
    _check(lib().tcu_translate(ctx.handle, count, _p(labels), _p(args), int(helicity), int(bool(singular)), _p(out)))
    out = out.reshape(shape)
    return complex(out) if out.ndim == 0 else out


def translate_block(lmax, k, displacement, singular=True, helicity=True, ctx=None):
    """All coefficients between the modes of one lmax basis (TranslationPlan::evaluate) as an
    (M, M) block, destination modes as rows."""
    return translation_block(lmax, k, displacement, singular, helicity, ctx)


def wigner3j(j1: int, j2: int, j3: int, m1: int, m2: int, m3: int) -> float:
    """Wigner 3j symbol (special.wigner3j; treams-core special/wigner.rs:263), degrees <= 60,
    from the library's binary128 Racah formula (the one its translation plans use)."""
    return float(lib().tcu_wigner3j(int(j1), int(j2), int(j3), int(m1), int(m2), int(m3)))
