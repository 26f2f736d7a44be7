"""GPU parity of the cluster path against the CPU oracle (same seeded inputs).

Tolerances: translation blocks, Mie blocks and plane-wave coefficients within 1e-12 of
the block's scale; dense solves within 1e-10 relative in the scattered coefficients and
the cross sections; FP64 residual certificates <= 1e-13 |T b| for the
mixed path.
"""
import numpy as np
import pytest

import oracle
from test_oracle import translation_identities
from treams_b200 import workloads

pytestmark = pytest.mark.gpu


def rel(a, b):
    return np.linalg.norm(np.asarray(a) - np.asarray(b)) / np.linalg.norm(np.asarray(b))


@pytest.mark.parametrize("L", [3, 4, 6])
@pytest.mark.parametrize("singular", [True, False])
def test_translation_block_matches_oracle(ctx, L, singular):
    import treams_b200 as t
    for d, k in [([0.7, -0.4, 1.1], 1.3), ([0.0, 0.0, 0.45], 2.0), ([0.2, 0.1, -0.05], 1.5), ([3.0, -2.0, 0.5], 3.1)]:
        g = t.translation_block(L, k, d, singular=singular, ctx=ctx)
        o = oracle.translation_block(L, k, d, singular=singular)
        assert np.abs(g - o).max() <= 1e-12 * np.abs(o).max(), (d, k)
    pb = t.translation_block(3, 1.3, [0.4, 0.2, -0.3], singular=True, helicity=False, ctx=ctx)
    assert pb.shape == (30, 30)


def test_translation_block_identities(ctx):
    import treams_b200 as t
    fn = lambda L, d: t.translation_block(L, 1.7, d, ctx=ctx)  # noqa: E731
    assert translation_identities(fn, 4, [0.6, -0.2, 0.9]) <= 1e-12


def test_mie_blocks_match_oracle(ctx):
    import treams_b200 as t
    radii = np.array([0.1, 0.2, 0.3, 0.25])
    eps = np.array([4 + 0.1j, 2.25 + 0.01j, 9.0, 6 + 0.2j])
    for k0 in (0.5, 1.3, 3.0):
        g = t.mie_blocks(6, k0, radii, eps, ctx=ctx)
        for i in range(4):
            for l in range(1, 7):
                o = oracle.mie_block(l, k0 * radii[i], complex(eps[i]))
                assert np.abs(g[i, l - 1] - o).max() <= 1e-12 * np.abs(o).max() + 1e-300


def test_plane_wave_matches_oracle(ctx):
    import treams_b200 as t
    w = workloads.precision_cluster(count=16)
    g = t.plane_wave_expansion(4, w.positions, w.kvecs, w.pols, ctx=ctx)
    o = oracle.plane_wave_expansion(4, w.positions, w.kvecs, w.pols)
    assert rel(g, o) <= 1e-13


def test_operator_matches_oracle_small_cluster(ctx):
    import treams_b200 as t
    w = workloads.small_cluster()
    g = t.cluster_operator(w.lmax, w.k0, w.radii, w.eps, w.positions, ctx=ctx)
    o, _ = oracle.cluster_operator(w.lmax, w.k0, w.radii, w.eps, w.positions)
    assert np.abs(g - o).max() <= 1e-12 * np.abs(o).max()


def test_operator_matches_oracle_lmax4_subset(ctx):
    import treams_b200 as t
    w = workloads.precision_cluster(count=40)
    g = t.cluster_operator(w.lmax, w.k0, w.radii, w.eps, w.positions, ctx=ctx)
    o, _ = oracle.cluster_operator(w.lmax, w.k0, w.radii, w.eps, w.positions)
    assert np.abs(g - o).max() <= 1e-12 * np.abs(o).max()


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_dense_solve_small_cluster(ctx, precision):
    import treams_b200 as t
    w = workloads.small_cluster()
    A, tb = oracle.cluster_operator(w.lmax, w.k0, w.radii, w.eps, w.positions)
    B = oracle.plane_wave_expansion(w.lmax, w.positions, w.kvecs, w.pols)
    Xo = oracle.dense_solve(w.lmax, A, tb, B)
    f = t.sphere_cluster_factor(w.lmax, w.k0, w.radii, w.eps, w.positions, precision, ctx=ctx)
    X, certs = f.solve(B)
    assert rel(X, Xo) <= 1e-10
    so, eo = oracle.cross_sections(w.lmax, w.k0, w.positions, Xo[:, 0], B[:, 0])
    sg, eg = t.cross_sections(w.lmax, w.k0, w.positions, X, B, ctx=ctx)
    assert abs(sg[0] - so) <= 1e-10 * abs(so) and abs(eg[0] - eo) <= 1e-10 * abs(eo)
    assert certs[0].residual_norm <= 1e-12 * certs[0].rhs_norm


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_dense_solve_lmax4_subset(ctx, precision):
    # 64 spheres of the 512-sphere precision workload's distribution (n = 3072), 3 columns
    import treams_b200 as t
    w = workloads.precision_cluster(count=64)
    A, tb = oracle.cluster_operator(w.lmax, w.k0, w.radii, w.eps, w.positions)
    B = oracle.plane_wave_expansion(w.lmax, w.positions, w.kvecs, w.pols)
    TB = np.zeros_like(B)
    M = 48
    ls = [l for l in range(1, 5) for _ in range(2 * l + 1)]
    for i in range(64):
        for q, l in enumerate(ls):
            TB[i * M + 2 * q:i * M + 2 * q + 2] = tb[i, l - 1] @ B[i * M + 2 * q:i * M + 2 * q + 2]
    Xo = np.linalg.solve(A, TB)
    f = t.sphere_cluster_factor(w.lmax, w.k0, w.radii, w.eps, w.positions, precision, ctx=ctx)
    X, certs = f.solve(B)
    assert rel(X, Xo) <= 1e-10
    for c in certs:
        assert c.residual_norm <= 1e-12 * c.rhs_norm
        # an FP32-accurate factor reaches 1e-13 in a handful of FP64 refinement sweeps
        assert c.iterations <= (1 if precision == "fp64" else 5)


def test_lossless_energy_balance_on_gpu(ctx):
    import treams_b200 as t
    w = workloads.small_cluster()
    eps = np.full(8, 4.0 + 0j)
    f = t.sphere_cluster_factor(w.lmax, w.k0, w.radii, eps, w.positions, "fp64", ctx=ctx)
    B = t.plane_wave_expansion(w.lmax, w.positions, w.kvecs, w.pols, ctx=ctx)
    X, _ = f.solve(B)
    sca, ext = t.cross_sections(w.lmax, w.k0, w.positions, X, B, ctx=ctx)
    assert sca[0] == pytest.approx(ext[0], rel=1e-12)


def test_matrix_free_apply_and_gmres_match_oracle(ctx):
    import treams_b200 as t
    w = workloads.small_cluster()
    rng = np.random.default_rng(5)
    x = rng.standard_normal((w.n, 3)) + 1j * rng.standard_normal((w.n, 3))
    yg = t.cluster_apply(w.lmax, w.k0, w.radii, w.eps, w.positions, x, ctx=ctx)
    yo = oracle.iterative_apply(w.lmax, w.k0, w.radii, w.eps, w.positions, x)
    assert rel(yg, yo) <= 1e-13
    B = oracle.plane_wave_expansion(w.lmax, w.positions, w.kvecs, w.pols)
    Xo, its, res, st = oracle.iterative_solve(w.lmax, w.k0, w.radii, w.eps, w.positions, B)
    sol = t.SphereCluster(w.lmax, w.k0, w.radii, w.eps, w.positions, ctx=ctx).solve(B)
    assert rel(sol.value, Xo) <= 2e-10
    c = sol.convergence[0]
    assert c.residual_norm <= 1e-10 * c.rhs_norm


def test_invalid_inputs_raise(ctx):
    import treams_b200 as t
    with pytest.raises(ValueError, match="touch or overlap"):
        t.sphere_cluster_factor(3, 1.0, [0.5, 0.5], [4, 4], [[0, 0, 0], [0.9, 0, 0]], ctx=ctx)
    with pytest.raises(ValueError, match="positive finite k0"):
        t.sphere_cluster_factor(3, -1.0, [0.5], [4], [[0, 0, 0]], ctx=ctx)
    with pytest.raises(ValueError, match="GMRES needs"):
        t.SphereCluster(3, 1.0, [0.5], [4], [[0, 0, 0]], ctx=ctx).solve(np.ones(30), rtol=0.0, atol=0.0)


def test_touching_pair_is_found_among_many_spheres(ctx):
    # the cell-grid validation must find an overlapping pair wherever it sits in the list
    import treams_b200 as t
    g = np.stack(np.meshgrid(np.arange(6), np.arange(6), np.arange(6), indexing="ij"), -1).reshape(-1, 3) * 0.7
    radii = np.full(len(g), 0.3)
    ok = t.cluster_apply(1, 1.0, radii, np.full(len(g), 2.0 + 0j), g, np.ones(len(g) * 6, complex), ctx=ctx)
    assert np.all(np.isfinite(ok))
    bad = g.copy()
    bad[150] = bad[3] + np.array([0.55, 0.1, 0.0])  # 0.559 < 0.6: overlaps sphere 3
    with pytest.raises(ValueError, match="touch or overlap"):
        t.cluster_apply(1, 1.0, radii, np.full(len(g), 2.0 + 0j), bad, np.ones(len(g) * 6, complex), ctx=ctx)
