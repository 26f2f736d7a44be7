"""The CPU oracle against the reference's golden tables and oracle-independent identities."""
import numpy as np
import pytest

import oracle
from conftest import read_table

from treams_b200 import workloads


def test_hankel_matches_high_precision_table():
    # crates/treams-core/src/special/bessel.rs:715-734: within 1e-13 of 90-digit values
    rows = read_table("spherical_hankel.txt")
    assert len(rows) == 6
    for key, val in rows:
        l, x = int(key[0]), float(key[1])
        h = oracle.spherical_hankels(l, x)[l]
        e = complex(float(val[0]), float(val[1]))
        assert abs(h - e) <= 1e-13 * abs(e), (l, x, h, e)


def test_small_argument_hankel_agrees_with_recurrence():
    # below x = 0.5 the oracle takes j_l by series + y_l upward; it must agree with the
    # plain recurrence (which is accurate in norm there) to 1e-13 relative
    for x in (0.1, 0.3, 0.49):
        h1 = oracle.spherical_h(12, complex(x, 0))
        xs = x
        prev, cur = np.exp(1j * xs) / xs, -1j * np.exp(1j * xs) / xs
        for l in range(13):
            assert abs(h1[l] - cur) <= 1e-13 * abs(cur)
            prev, cur = cur, (2 * l + 1) / xs * cur - prev


def test_degrees_match_lean_model():
    # coupling.rs:192-217 against formal/golden/degrees.txt
    rows = read_table("degrees.txt")
    assert len(rows) == 2450
    for key, vals in rows:
        l, m, lam, mu, cross = map(int, key)
        assert oracle.degrees(l, m, lam, mu, cross) == [int(v) for v in vals], key


def test_harmonic_table_order():
    # plan.rs:939-963 against formal/golden/harmonics.txt: (p, m) at p*p+p+m
    for key, vals in read_table("harmonics.txt"):
        lmax = int(key[0])
        pairs = [tuple(map(int, v.split(","))) for v in vals]
        expected = [(p, m) for p in range(lmax + 1) for m in range(-p, p + 1)]
        assert pairs == expected
        for idx, (p, m) in enumerate(pairs):
            assert p * p + p + m == idx


def test_wigner3j_known_values_and_orthogonality():
    assert oracle.wigner3j(1, 1, 0, 0, 0, 0) == pytest.approx(-1 / np.sqrt(3), abs=1e-15)
    assert oracle.wigner3j(2, 2, 2, 0, 0, 0) == pytest.approx(-np.sqrt(2 / 35), abs=1e-15)
    # sum_{j3, m3} (2 j3 + 1) (j1 j2 j3; m1 m2 m3)^2 = 1
    for j1, j2, m1, m2 in [(3, 5, 1, -2), (6, 6, 0, 0), (4, 7, -3, 2)]:
        s = sum((2 * j3 + 1) * oracle.wigner3j(j1, j2, j3, m1, m2, -m1 - m2) ** 2 for j3 in range(0, j1 + j2 + 1))
        assert s == pytest.approx(1.0, abs=1e-13)


def test_regular_translation_at_origin_is_identity():
    # plan.rs:669-685
    for L in (3, 4, 6):
        B = oracle.translation_block(L, 1.7, [0.0, 0.0, 0.0], singular=False)
        assert np.abs(B - np.eye(B.shape[0])).max() < 1e-13


def translation_identities(block_fn, L, d, angle=0.7):
    """Parity, reciprocity and azimuthal covariance of sw/plan.rs:725-800 (helicity modes):
    A(-d)[to, from] = (-1)^(l+lambda) A(d)[flip to, flip from];
    A(d)[(lam,mu,t), (l,m,s)] = (-1)^(m+mu) A(-d)[(l,-m,s), (lam,-mu,t)];
    A(R_z d)[to, from] = e^{i (m - mu) angle} A(d)[to, from]."""
    md = oracle.modes(L)
    index = {mode: i for i, mode in enumerate(md)}
    A = block_fn(L, d)
    B = block_fn(L, -np.asarray(d))
    c, s = np.cos(angle), np.sin(angle)
    R = block_fn(L, [d[0] * c - d[1] * s, d[0] * s + d[1] * c, d[2]])
    scale = np.abs(A).max()
    worst = 0.0
    for ti, (lam, mu, t) in enumerate(md):
        for fi, (l, m, s_) in enumerate(md):
            flip = A[index[(lam, mu, 1 - t)], index[(l, m, 1 - s_)]] * (-1.0) ** (l + lam)
            worst = max(worst, abs(B[ti, fi] - flip))
            rec = (-1.0) ** (m + mu) * B[index[(l, -m, s_)], index[(lam, -mu, t)]]
            worst = max(worst, abs(A[ti, fi] - rec))
            rot = np.exp(1j * (m - mu) * angle) * A[ti, fi]
            worst = max(worst, abs(R[ti, fi] - rot))
    return worst / scale


def test_translation_parity_reciprocity_rotation():
    fn = lambda L, d: oracle.translation_block(L, 1.3, d)  # noqa: E731
    assert translation_identities(fn, 3, [0.7, -0.4, 1.1]) <= 1e-12
    assert translation_identities(fn, 4, [-0.3, 0.9, 0.2]) <= 1e-12


def test_plan_term_count_within_degree_bound():
    # the survey's per-block upper bounds from `degrees`
    for L, bound in ((3, 1578), (4, 4904), (5, 12302), (6, 26700)):
        assert 0 < oracle.plan_terms(L) <= bound


def test_lossless_cluster_conserves_energy():
    # properties/tmatrix.rs:203: sigma_ext = sigma_sca without absorption
    w = workloads.small_cluster()
    eps = np.full(8, 4.0 + 0j)
    A, tb = oracle.cluster_operator(w.lmax, w.k0, w.radii, eps, w.positions)
    B = oracle.plane_wave_expansion(w.lmax, w.positions, w.kvecs, w.pols)
    X = oracle.dense_solve(w.lmax, A, tb, B)
    sca, ext = oracle.cross_sections(w.lmax, w.k0, w.positions, X[:, 0], B[:, 0])
    assert sca == pytest.approx(ext, rel=1e-12)
    assert sca > 0


def test_lu_matches_lapack_and_gmres_matches_dense():
    rng = np.random.default_rng(7)
    n = 120
    A = np.eye(n) * 3 + (rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))) / np.sqrt(n)
    b = rng.standard_normal((n, 2)) + 1j * rng.standard_normal((n, 2))
    x = oracle.lu_solve(A, b)
    assert np.linalg.norm(x - np.linalg.solve(A, b)) <= 1e-13 * np.linalg.norm(x)
    xg, its, res, st = oracle.gmres_dense(A, b[:, 0], rtol=1e-12, restart=8, max_iterations=200)
    assert st == 0 and res <= 1e-12 * np.linalg.norm(b[:, 0])
    assert np.linalg.norm(xg - x[:, 0]) <= 1e-10 * np.linalg.norm(x[:, 0])


def test_matrix_free_equals_dense_and_gmres_converges():
    # cluster/iterative.rs:714-846
    w = workloads.small_cluster()
    A, tb = oracle.cluster_operator(w.lmax, w.k0, w.radii, w.eps, w.positions)
    rng = np.random.default_rng(3)
    x = rng.standard_normal((A.shape[0], 2)) + 1j * rng.standard_normal((A.shape[0], 2))
    y = oracle.iterative_apply(w.lmax, w.k0, w.radii, w.eps, w.positions, x)
    assert np.linalg.norm(y - A @ x) <= 1e-13 * np.linalg.norm(A @ x)
    B = oracle.plane_wave_expansion(w.lmax, w.positions, w.kvecs, w.pols)
    X = oracle.dense_solve(w.lmax, A, tb, B)
    Xi, its, res, st = oracle.iterative_solve(w.lmax, w.k0, w.radii, w.eps, w.positions, B)
    assert st == 0
    assert np.linalg.norm(Xi - X) <= 2e-10 * np.linalg.norm(X)


def test_single_sphere_reduces_to_mie():
    # iterative.rs:762-772: one sphere, the cluster solve is T b
    k0, r, eps = 1.1, 0.4, 3.0 + 0.2j
    A, tb = oracle.cluster_operator(3, k0, [r], [eps], [[0.2, -0.1, 0.3]])
    assert np.abs(A - np.eye(30)).max() == 0.0
    b = np.ones((30, 1), complex)
    X = oracle.dense_solve(3, A, tb, b)
    Tb = np.concatenate([tb[0, l - 1] @ b[2 * q:2 * q + 2, 0] for l, q in
                         [(l, i) for i, l in enumerate([l for l in range(1, 4) for _ in range(2 * l + 1)])]])
    assert np.allclose(X[:, 0], Tb, rtol=0, atol=1e-15)


def test_network_restatement_with_theta_one_is_the_near_field_neumann_term():
    # all output weights zero: Theta = 1 and M r = r + T C_near r, with C_near the coupling
    # blocks of the pairs within 3 sphere diameters (the dense oracle operator, masked)
    w = workloads.learned_cluster(seed=91, count=12)
    A, tb = oracle.cluster_operator(w.lmax, w.k0, w.radii, w.eps, w.positions)
    lay, total = oracle.gnn_layout(w.lmax)
    rng = np.random.default_rng(1)
    W = rng.standard_normal(total) * 0.3
    W[lay["W4"][0]:] = 0.0
    R = rng.standard_normal((w.n, 2)) + 1j * rng.standard_normal((w.n, 2))
    D = np.linalg.norm(w.positions[:, None] - w.positions[None], axis=2)
    M = 2 * w.lmax * (w.lmax + 2)
    near = np.kron((D <= 1.2) & (D > 0), np.ones((M, M), bool))
    TC_near = np.where(near, np.eye(w.n) - A, 0.0)
    expected = np.sum(np.abs(R - A @ (R + TC_near @ R)) ** 2)
    got = oracle.gnn_loss(w.lmax, w.k0, w.radii, w.eps, w.positions, R, W, A=A, tb=tb)
    assert got == pytest.approx(expected, rel=1e-12)
