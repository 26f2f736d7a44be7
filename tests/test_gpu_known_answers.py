"""GPU results against the reference's own known answers (tests/golden/known_answers.txt and
closed forms written in the reference's tests).

- Mie blocks of the metallic sphere x = 80, eps = -8 + 0.4i at l = 1 and 3
  (crates/treams-core/src/coeffs/mie.rs:573-612), tolerance 2e-13 + 2e-11 |v| as there;
- the closed dipole forms of A(1,0;1,1) and B(1,0;1,1), outgoing and regular, at the complex
  argument z = 1.4 + 0.2i and polar angles down to 1e-100 (tests/waves/
  test_translation_coefficients.py:63-88), rtol 3e-13 as there, through the per-entry
  sw.translate of the library;
- the per-entry coefficients equal the entries of the oracle's translation blocks at real
  arguments (relative 1e-12 of the block's scale).
"""
import numpy as np
import pytest

import oracle
from conftest import read_table

pytestmark = pytest.mark.gpu


def test_gpu_mie_matches_metallic_sphere_known_answers(ctx):
    import treams_b200 as t
    rows = [(k[1:], [float(v) for v in vals]) for k, vals in read_table("known_answers.txt") if k[0] == "mie"]
    checked = 0
    for key, v in rows:
        l, x, er, ei = int(key[0]), float(key[1]), float(key[2]), float(key[3])
        if l > 7:  # the device Mie kernel serves degrees <= 7; the oracle test covers 80 and 99
            continue
        blocks = t.mie_blocks(l, 1.0, [x], [complex(er, ei)], ctx=ctx)[0, l - 1]
        diag, off = complex(v[0], v[1]), complex(v[2], v[3])
        expected = np.array([[diag, off], [off, diag]])
        for a, e in zip(blocks.ravel(), expected.ravel()):
            assert abs(a - e) <= 2e-13 + 2e-11 * abs(e), (l, a, e)
        checked += 1
    assert checked == 2


@pytest.mark.parametrize("regular", [False, True])
def test_dipole_translation_matches_closed_form_at_complex_argument(ctx, regular):
    from treams_b200 import sw
    z = 1.4 + 0.2j
    h1 = -np.exp(1j * z) * (z + 1j) / z**2
    h2 = np.exp(1j * z) * (1j / z - 3 / z**2 - 3j / z**3)
    j1 = np.sin(z) / z**2 - np.cos(z) / z
    j2 = (3 / z**3 - 1 / z) * np.sin(z) - 3 * np.cos(z) / z**2
    r1, r2 = (j1, j2) if regular else (h1, h2)
    for theta in [1e-8, 1e-10, 1e-100]:
        phase = np.exp(0.4j) * np.sin(theta)
        expected_a = -3 / (2 * np.sqrt(2)) * r2 * np.cos(theta) * phase
        expected_b = 3j / (2 * np.sqrt(2)) * r1 * phase
        # parity modes: equal parities give A, different ones B (destination (1, 0), source (1, 1))
        a = sw.translate(1, 0, 0, 1, 1, 0, z, theta, 0.4, poltype="parity", singular=not regular, ctx=ctx)
        b = sw.translate(1, 0, 0, 1, 1, 1, z, theta, 0.4, poltype="parity", singular=not regular, ctx=ctx)
        assert abs(a - expected_a) <= 3e-13 * abs(expected_a), (theta, a, expected_a)
        assert abs(b - expected_b) <= 3e-13 * abs(expected_b), (theta, b, expected_b)
        # helicity modes: A +- B for equal helicities, 0 across
        hp = sw.translate(1, 0, 1, 1, 1, 1, z, theta, 0.4, singular=not regular, ctx=ctx)
        hm = sw.translate(1, 0, 0, 1, 1, 0, z, theta, 0.4, singular=not regular, ctx=ctx)
        hx = sw.translate(1, 0, 1, 1, 1, 0, z, theta, 0.4, singular=not regular, ctx=ctx)
        assert abs(hp - (expected_a + expected_b)) <= 3e-13 * abs(expected_a + expected_b)
        assert abs(hm - (expected_a - expected_b)) <= 3e-13 * abs(expected_a - expected_b)
        assert hx == 0


@pytest.mark.parametrize("L", [3, 5])
@pytest.mark.parametrize("singular", [True, False])
def test_per_entry_translate_equals_oracle_blocks(ctx, L, singular):
    from treams_b200 import sw
    md = oracle.modes(L)
    for d, k in [([0.7, -0.4, 1.1], 1.3), ([0.2, 0.1, -0.05], 1.5), ([-2.0, 0.3, -0.6], 2.2)]:
        block = oracle.translation_block(L, k, d, singular=singular, helicity=True)
        r = np.linalg.norm(d)
        theta, phi = np.arccos(d[2] / r), np.arctan2(d[1], d[0])
        lam, mu, pol = (np.array([m[i] for m in md])[:, None] for i in range(3))
        l, m, qol = (np.array([m_[i] for m_ in md])[None, :] for i in range(3))
        vals = sw.translate(lam, mu, pol, l, m, qol, k * r, theta, phi, singular=singular, ctx=ctx)
        assert vals.shape == block.shape
        assert np.abs(vals - block).max() <= 1e-12 * np.abs(block).max(), (d, k)


def test_translate_rejects_bad_labels(ctx):
    from treams_b200 import sw
    with pytest.raises(ValueError, match="mode labels"):
        sw.translate(0, 0, 1, 1, 0, 1, 1.0, 0.3, 0.1, ctx=ctx)
    assert sw.translate(1, 0, 1, 1, 0, 1, 0.0, 0.3, 0.1, ctx=ctx) == 0  # singular self term


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_gpu_sic_chain_absorption_matches_the_known_answer(ctx, precision):
    # tests/tmatrix/test_particle_cluster.py:539-562: lmax 10, entries of I - T C near 1e22
    import treams_b200 as t
    from test_known_answers import absorption, sic_chain
    L, k0, radii, eps, pos = sic_chain()
    value, rtol = [float(v) for v in next(v for k, v in read_table("known_answers.txt")
                                          if k[0] == "sic_chain_absorption_1e12")]
    f = t.sphere_cluster_factor(L, k0, radii, eps, pos, precision, ctx=ctx)
    try:
        Tg = f.global_tmatrix(10)
    finally:
        f.close()
    assert absorption(Tg, k0) * 1e12 == pytest.approx(value, rel=rtol)
    orders = np.array([m for (l, m, p) in oracle.modes(L)])
    assert np.abs(Tg[orders[:, None] != orders[None, :]]).max() <= 2e-20


def test_interacting_tmatrix_matches_dense_solve(ctx):
    import treams_b200 as t
    from treams_b200 import workloads
    w = workloads.small_cluster()
    A, tb = oracle.cluster_operator(w.lmax, w.k0, w.radii, w.eps, w.positions)
    Xo = np.linalg.solve(A, oracle.apply_t(w.lmax, tb, np.eye(w.n)))
    f = t.sphere_cluster_factor(w.lmax, w.k0, w.radii, w.eps, w.positions, "fp64", ctx=ctx)
    try:
        X = f.interacting_tmatrix()
        Tg = f.global_tmatrix(3, origin=w.positions.mean(axis=0))
    finally:
        f.close()
    assert np.linalg.norm(X - Xo) <= 1e-10 * np.linalg.norm(Xo)
    # the global T-matrix: sum_ij R(o <- r_i) X_ij R(r_j <- o) with the oracle's blocks
    M, o = 30, w.positions.mean(axis=0)
    Tgo = np.zeros((M, M), complex)
    for i in range(8):
        Ri = oracle.translation_block(3, w.k0, o - w.positions[i], singular=False)
        for j in range(8):
            Tgo += Ri @ Xo[i * M:(i + 1) * M, j * M:(j + 1) * M] @ oracle.translation_block(
                3, w.k0, w.positions[j] - o, singular=False)
    assert np.linalg.norm(Tg - Tgo) <= 1e-10 * np.linalg.norm(Tgo)
