"""Spherical-wave translations (treams_rs.sw)."""
from ._lib import modes, translation_block  # noqa: F401


def translate_block(lmax, k, displacement, singular=True, helicity=True, ctx=None):
    """Translation coefficients of a whole mode block (sw.translate over a basis)."""
    return translation_block(lmax, k, displacement, singular, helicity, ctx)
