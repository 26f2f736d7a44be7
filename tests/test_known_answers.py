"""The reference's own known answers, read from its test sources into tests/golden/known_answers.txt
(tests/golden/make_fixtures.py), against the CPU oracle and the library's host-side Wigner 3j.

- Mie blocks of a metallic sphere, x = 80, eps = -8 + 0.4i, l = 1, 3, 80, 99
  (crates/treams-core/src/coeffs/mie.rs:573-612), tolerance 2e-13 + 2e-11 |v| as there;
- the 30-digit symbol (15 15 23; 15 -15 0) in its three even argument orders
  (tests/special/test_wigner.py:114-122), rtol 1e-12 as there.
No GPU is needed: the oracle is C++ and tcu_wigner3j is host code of the library.
"""
import numpy as np
import pytest

import oracle
from conftest import read_table


def _rows(kind):
    return [(k[1:], [float(v) for v in vals]) for k, vals in read_table("known_answers.txt") if k[0] == kind]


def test_known_answer_table_is_complete():
    assert len(_rows("mie")) == 4 and len(_rows("wigner3j")) == 1 and any(k[0] == "sic_chain_absorption_1e12" for k, _ in read_table("known_answers.txt"))


@pytest.mark.parametrize("row", range(4))
def test_oracle_mie_matches_metallic_sphere_known_answers(row):
    key, v = _rows("mie")[row]
    l, x, er, ei = int(key[0]), float(key[1]), float(key[2]), float(key[3])
    diag, off = complex(v[0], v[1]), complex(v[2], v[3])
    block = oracle.mie_block(l, x, complex(er, ei))
    expected = np.array([[diag, off], [off, diag]])
    for a, e in zip(block.ravel(), expected.ravel()):
        assert abs(a - e) <= 2e-13 + 2e-11 * abs(e), (l, a, e)


def _wigner_cases():
    key, v = _rows("wigner3j")[0]
    j1, j2, j3, m1, m2, m3 = map(int, key)
    # the even permutations of the symbol keep its value
    return [((j1, j2, j3, m1, m2, m3), v[0]), ((j3, j1, j2, m3, m1, m2), v[0]), ((j2, j3, j1, m2, m3, m1), v[0])]


@pytest.mark.parametrize("case", range(3))
def test_oracle_wigner3j_matches_the_30_digit_value(case):
    args, value = _wigner_cases()[case]
    assert oracle.wigner3j(*args) == pytest.approx(value, rel=1e-12)


@pytest.mark.parametrize("case", range(3))
def test_library_racah_wigner3j_matches_the_30_digit_value(case):
    # the binary128 Racah formula that builds every translation plan of the library
    from treams_b200 import sw
    args, value = _wigner_cases()[case]
    assert sw.wigner3j(*args) == pytest.approx(value, rel=1e-14)


def test_library_wigner3j_agrees_with_the_oracle_recurrence():
    from treams_b200 import sw
    rng = np.random.default_rng(4)
    for _ in range(300):
        j1, j2 = rng.integers(0, 16, 2)
        j3 = int(rng.integers(abs(j1 - j2), j1 + j2 + 1))
        m1 = int(rng.integers(-j1, j1 + 1))
        m2 = int(rng.integers(-j2, j2 + 1))
        m3 = -m1 - m2
        if abs(m3) > j3:
            continue
        a, b = sw.wigner3j(j1, j2, j3, m1, m2, m3), oracle.wigner3j(j1, j2, j3, m1, m2, m3)
        assert abs(a - b) <= 1e-13 * max(1.0, abs(b)) and abs(a - b) <= 2e-14 + 1e-11 * abs(b)


def sic_chain():
    """Four 250 nm SiC spheres with 20 nm gaps on the z axis at 3 THz, lmax 10
    (tests/tmatrix/test_particle_cluster.py:539-562)."""
    k0 = 2 * np.pi * 3e12 / 299792458.0
    pos = np.array([[0.0, 0.0, z * 520e-9] for z in (-1.5, -0.5, 0.5, 1.5)])
    return 10, k0, np.full(4, 250e-9), np.full(4, 12.87707323 + 0.19225647000000007j), pos


def absorption(Tg, k0):
    return -2 * np.pi * (np.trace(Tg).real + np.vdot(Tg, Tg).real) / k0**2


def test_oracle_sic_chain_absorption_matches_the_known_answer():
    # I - T C has a unit diagonal but entries near 1e22 at degree 10: the solve equilibrates
    # rows and columns by powers of two (as the library's factorization does), then the
    # cluster T-matrix is expanded into the lmax-10 basis at the origin with regular
    # translations: T_g = sum_ij R(0 <- r_i) X_ij R(r_j <- 0)
    import scipy.linalg
    L, k0, radii, eps, pos = sic_chain()
    value, rtol = [float(v) for v in next(v for k, v in read_table("known_answers.txt")
                                          if k[0] == "sic_chain_absorption_1e12")]
    A, tb = oracle.cluster_operator(L, k0, radii, eps, pos)
    M = 2 * L * (L + 2)
    n = 4 * M
    T = oracle.apply_t(L, tb, np.eye(n))
    R = 2.0 ** -np.round(np.log2(np.abs(A).max(axis=1)))
    A1 = A * R[:, None]
    C = 2.0 ** -np.round(np.log2(np.abs(A1).max(axis=0)))
    X = C[:, None] * scipy.linalg.solve(A1 * C[None, :], R[:, None] * T)
    Tg = np.zeros((M, M), complex)
    for i in range(4):
        Ri = oracle.translation_block(L, k0, -pos[i], singular=False)
        for j in range(4):
            Tg += Ri @ X[i * M:(i + 1) * M, j * M:(j + 1) * M] @ oracle.translation_block(L, k0, pos[j], singular=False)
    assert absorption(Tg, k0) * 1e12 == pytest.approx(value, rel=rtol)
    orders = np.array([m for (l, m, p) in oracle.modes(L)])
    assert np.abs(Tg[orders[:, None] != orders[None, :]]).max() <= 2e-20
