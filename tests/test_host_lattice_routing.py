"""Host logic of the lattice-sum wrapper (no GPU): which C-ABI entry point a call reaches and
what it passes. A real k without a shift takes tcu_lsumsw2d_batch, with a shift
tcu_lsumsw2d_shift_batch, and a complex k (a lossy embedding) tcu_lsumsw2d_complex_batch with
k as (re, im) and a zero shift when none is given."""
import ctypes

import numpy as np

from treams_b200 import lattice as tl


def _doubles(addr, n):
    return list((ctypes.c_double * n).from_address(addr))


class _FakeLib:
    def __init__(self):
        self.calls = []

    def tcu_lsumsw2d_batch(self, handle, lmax_sum, k, lattice, nk, kpars, eta, out):
        self.calls.append(("plain", lmax_sum, k, nk, eta, None))
        return 0

    def tcu_lsumsw2d_shift_batch(self, handle, lmax_sum, k, lattice, nk, kpars, shift, eta, out):
        self.calls.append(("shift", lmax_sum, k, nk, eta, _doubles(shift, 3)))
        return 0

    def tcu_lsumsw2d_complex_batch(self, handle, lmax_sum, k, lattice, nk, kpars, shift, eta, out):
        self.calls.append(("complex", lmax_sum, _doubles(k, 2), nk, eta, _doubles(shift, 3)))
        return 0


class _FakeContext:
    handle = None


def _call(monkeypatch, *args, **kwargs):
    fake = _FakeLib()
    monkeypatch.setattr(tl, "lib", lambda: fake)
    out = tl.lsumsw2d_batch(*args, ctx=_FakeContext(), **kwargs)
    assert len(fake.calls) == 1
    return out, fake.calls[0]


def test_real_wavenumber_without_shift(monkeypatch):
    out, call = _call(monkeypatch, 4, 2.5, np.eye(2), [[0.1, 0.2], [0.3, 0.4], [0.0, 0.0]])
    assert call == ("plain", 4, 2.5, 3, 0.0, None)
    assert out.shape == (3, 25) and out.dtype == np.complex128


def test_real_wavenumber_with_a_shift_off_the_plane(monkeypatch):
    _, call = _call(monkeypatch, 6, 2.5, np.eye(2), [[0.1, 0.2]], eta=0.8, shift=(0.1, -0.2, 0.3))
    assert call == ("shift", 6, 2.5, 1, 0.8, [0.1, -0.2, 0.3])


def test_a_complex_value_with_zero_imaginary_part_stays_on_the_real_path(monkeypatch):
    _, call = _call(monkeypatch, 2, 2.5 + 0j, np.eye(2), [[0.1, 0.2]])
    assert call[0] == "plain" and call[2] == 2.5


def test_complex_wavenumber_without_and_with_a_shift(monkeypatch):
    _, call = _call(monkeypatch, 8, 2.7 + 0.4j, np.eye(2), [[0.1, 0.2], [0.5, 0.5]])
    assert call == ("complex", 8, [2.7, 0.4], 2, 0.0, [0.0, 0.0, 0.0])
    _, call = _call(monkeypatch, 8, 2.7 + 0.4j, np.eye(2), [[0.1, 0.2]], eta=0.9, shift=[0.3, 0.1, 0.25])
    assert call == ("complex", 8, [2.7, 0.4], 1, 0.9, [0.3, 0.1, 0.25])
