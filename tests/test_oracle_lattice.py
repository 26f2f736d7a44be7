"""The Ewald lattice-sum oracle against the reference's high-precision tables and identities.

Tables (copied from crates/treams-core/references/ by tests/golden/make_fixtures.py):
incomplete gamma Gamma(n, z) (incgamma.txt, incgamma_zero.txt; special/integrals/gamma.rs),
Kambe integrals (kambe.txt; special/integrals/kambe.rs) and the 2D spherical lattice sums
of lattice_sums.txt (lattice/mod.rs:283; the reference checks them in
`sums_match_high_precision_references` to `tolerance * max(|S|, 1)`).
"""
import math

import numpy as np
import pytest

import oracle
from conftest import read_table

from treams_b200 import workloads


def _rel(a, b):
    return abs(a - b) / abs(b) if b != 0 else abs(a)


def test_incomplete_gamma_table():
    rows = read_table("incgamma.txt")
    assert len(rows) > 1000
    for key, val in rows:
        a, zr, zi = float(key[0]), float(key[1]), float(key[2])  # "-0.0" keeps its sign
        ref = complex(float(val[0]), float(val[1]))
        g = oracle.upper_gamma(a, complex(zr, zi))
        assert _rel(g, ref) <= 1e-13, (key, g, ref)


def test_incomplete_gamma_at_its_zero():
    # Gamma(n, z) next to its zero Gamma(2, -1) = 0: absolute accuracy, both sides of the cut
    for key, val in read_table("incgamma_zero.txt"):
        a, zr, zi = float(key[0]), float(key[1]), float(key[2])
        ref = complex(float(val[0]), float(val[1]))
        g = oracle.upper_gamma(a, complex(zr, zi))
        assert abs(g - ref) <= 1e-13 * max(abs(ref), 1e-290) or abs(g - ref) < 1e-300, (key, g, ref)


def test_kambe_table():
    rows = read_table("kambe.txt")
    assert len(rows) > 150
    for key, val in rows:
        n, zr, zi, eta = int(key[0]), float(key[1]), float(key[2]), float(key[3])
        ref = complex(float(val[0]), float(val[1]))
        v = oracle.kambe(n, complex(zr, zi), complex(eta, 0.0))
        assert _rel(v, ref) <= 1e-13, (key, v, ref)


def _lattice_rows():
    out = []
    for key, val in read_table("lattice_sums_2d.txt"):
        (_, l, m, dim, kr, ki, x, y, z, er, ei, a11, a12, a21, a22, b1, b2, part, jet, tol) = key
        out.append(dict(l=int(l), m=int(m), k=complex(float(kr), float(ki)), r=[float(x), float(y), float(z)],
                        eta=complex(float(er), float(ei)), lattice=[float(a11), float(a12), float(a21), float(a22)],
                        kpar=[float(b1), float(b2)], part=part, tol=float(tol),
                        ref=complex(float(val[0]), float(val[1]))))
    return out


@pytest.mark.parametrize("row", _lattice_rows(), ids=lambda r: f"l{r['l']}m{r['m']}k{r['k']}eta{r['eta']}{r['part']}")
def test_lattice_sums_match_high_precision_references(row):
    v = oracle.lsumsw2d(row["l"], row["m"], row["k"], row["lattice"], row["kpar"], row["r"], row["eta"], row["part"])
    assert abs(v - row["ref"]) <= row["tol"] * max(abs(row["ref"]), 1.0), (v, row["ref"])


def test_lattice_sums_do_not_depend_on_the_split():
    # lattice/mod.rs: the exact sum does not depend on eta (tests/lattice/test_lattice.py:300-308)
    w = workloads.periodic_array()
    for kp in w.kpars[:2]:
        d0 = oracle.lsumsw2d_table(12, w.k0, w.lattice, kp)
        for eta in (0.45, 0.9):
            d1 = oracle.lsumsw2d_table(12, w.k0, w.lattice, kp, eta=eta)
            assert np.max(np.abs(d1 - d0)) <= 1e-20 * max(1.0, np.max(np.abs(d0)))


def test_lattice_sums_are_bloch_periodic():
    # D depends on kpar only modulo the reciprocal lattice at shift 0 (lattice/mod.rs:38-44)
    w = workloads.periodic_array()
    g = 2 * math.pi / w.period
    kp = w.kpars[3]
    d0 = oracle.lsumsw2d_table(8, w.k0, w.lattice, kp)
    d1 = oracle.lsumsw2d_table(8, w.k0, w.lattice, kp + np.array([g, -2 * g]))
    # the shifted Bloch vector is rounded to binary64 before the sum: ~1e-16 |G| of kpar
    assert np.max(np.abs(d1 - d0)) <= 1e-13 * max(1.0, np.max(np.abs(d0)))


def test_in_plane_sums_vanish_for_odd_l_plus_m():
    w = workloads.periodic_array()
    d = oracle.lsumsw2d_table(12, w.k0, w.lattice, w.kpars[5])
    for l in range(13):
        for m in range(-l, l + 1):
            if (l + m) % 2:
                assert abs(d[l * l + l + m]) <= 1e-25 * max(1.0, np.max(np.abs(d)))


def test_array_solve_of_a_sparse_lattice_reduces_to_the_single_sphere():
    # X = (I - T S)^-1 T tends to the sphere's own T-matrix as the lattice sums vanish
    # (period 200 wavelengths / (2 pi): |S| ~ 1/(A k^2))
    lmax, k0, radius, eps = 2, 1.0, 0.2, 4.0 + 0.1j
    big = 200.0
    X = oracle.array_solve(lmax, k0, radius, eps, [big, 0.0, 0.0, big], [0.01, 0.02])
    M = 2 * lmax * (lmax + 2)
    T = np.zeros((M, M), complex)
    for c in range(0, M, 2):
        l = math.isqrt(c // 2 + 1)
        T[c:c + 2, c:c + 2] = oracle.mie_block(l, k0 * radius, eps)
    assert np.all(np.isfinite(X))
    assert np.max(np.abs(X - T)) <= 1e-3 * np.max(np.abs(T))
    assert np.max(np.abs(X - T)) > 0.0
