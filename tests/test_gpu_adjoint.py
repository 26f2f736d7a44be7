"""Adjoint solves on the GPU against dense FP64 algebra on the oracle's operator.

- tcu_factor_solve_adjoint: Y = (I - T C)^-H G (Lu::solve_adjoint_in_place, linalg/mod.rs:436)
  from the FP64 and mixed factors, refined in FP64: relative error <= 1e-10, residual
  certificate <= 1e-12;
- tcu_factor_pullback_incident: T^H (I - T C)^-H G (cluster/interaction.rs:221-227), same bar;
- tcu_iterative_pullback_incident: the same gradient by adjoint GMRES (cluster/iterative.rs:
  460-488, incident part) at rtol 1e-11: relative error <= 1e-9.
"""
import numpy as np
import pytest

import oracle
import treams_b200 as t
from treams_b200 import workloads

pytestmark = pytest.mark.gpu


def _reference(w, G):
    A, tb = oracle.cluster_operator(w.lmax, w.k0, w.radii, w.eps, w.positions)
    Y = np.linalg.solve(A.conj().T, G)
    th = np.conj(np.swapaxes(tb, 2, 3))  # T^H per 2 x 2 block
    return Y, oracle.apply_t(w.lmax, th, Y)


def _cotangent(n, p, seed):
    rng = np.random.default_rng(seed)
    return np.asfortranarray(rng.standard_normal((n, p)) + 1j * rng.standard_normal((n, p)))


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("count", [8, 64])
def test_factor_adjoint_solve_and_pullback_match_dense_algebra(ctx, precision, count):
    w = workloads.small_cluster() if count == 8 else workloads.precision_cluster(count=count)
    G = _cotangent(w.n, 3, 17)
    Yo, Po = _reference(w, G)
    f = t.sphere_cluster_factor(w.lmax, w.k0, w.radii, w.eps, w.positions, precision, ctx=ctx)
    try:
        Y, certs = f.solve_adjoint(G)
        assert np.linalg.norm(Y - Yo) <= 1e-10 * np.linalg.norm(Yo)
        for c in certs:
            assert c.residual_norm <= 1e-12 * c.rhs_norm
        Pg, _ = f.pullback_incident(G)
        assert np.linalg.norm(Pg - Po) <= 1e-10 * np.linalg.norm(Po)
    finally:
        f.close()


def test_iterative_pullback_matches_dense_algebra(ctx):
    w = workloads.small_cluster()
    G = _cotangent(w.n, 2, 18)
    _, Po = _reference(w, G)
    c = t.SphereCluster(w.lmax, w.k0, w.radii, w.eps, w.positions, ctx=ctx)
    sol = c.pullback_incident(G, rtol=1e-11)
    for cert in sol.convergence:
        assert cert.residual_norm <= 1e-11 * cert.rhs_norm
    assert np.linalg.norm(sol.value - Po) <= 1e-9 * np.linalg.norm(Po)


def test_adjoint_is_the_conjugate_transpose_of_the_operator(ctx):
    # <A x, y> = <x, A^H y> through the solves: <A^-1 b, g> = <b, A^-H g>
    w = workloads.precision_cluster(count=24)
    rng = np.random.default_rng(19)
    f = t.sphere_cluster_factor(w.lmax, w.k0, w.radii, w.eps, w.positions, "fp64", ctx=ctx)
    try:
        b = rng.standard_normal(w.n) + 1j * rng.standard_normal(w.n)
        g = rng.standard_normal(w.n) + 1j * rng.standard_normal(w.n)
        B = t.plane_wave_expansion(w.lmax, w.positions, w.kvecs, w.pols, ctx=ctx)
        X, _ = f.solve(B[:, :1])          # A^-1 T b
        Y, _ = f.solve_adjoint(g)          # A^-H g
        A, tb = oracle.cluster_operator(w.lmax, w.k0, w.radii, w.eps, w.positions)
        TB = oracle.apply_t(w.lmax, tb, B[:, :1])[:, 0]
        lhs = np.vdot(g, X[:, 0])
        rhs = np.vdot(Y, TB)
        assert abs(lhs - rhs) <= 1e-11 * abs(lhs)
        del b
    finally:
        f.close()


@pytest.mark.parametrize("lmax", [2, 3, 4, 5])
def test_iterative_pullback_with_stored_tables_matches_the_on_the_fly_product(ctx, lmax, monkeypatch):
    # adjoint GMRES applies C from the pair tables stored once per call (default) or in
    # product form every time (TCU_APPLY=fly)
    w = workloads.learned_cluster(seed=160 + lmax, count=120)
    n = w.radii.size * 2 * lmax * (lmax + 2)
    G = _cotangent(n, 2, 20 + lmax)
    c = t.SphereCluster(lmax, w.k0, w.radii, w.eps, w.positions, ctx=ctx)
    monkeypatch.delenv("TCU_APPLY", raising=False)
    s1 = c.pullback_incident(G, rtol=1e-12, restart=40, max_iterations=400)
    monkeypatch.setenv("TCU_APPLY", "fly")
    s2 = c.pullback_incident(G, rtol=1e-12, restart=40, max_iterations=400)
    # the two products differ by rounding only, so GMRES may stop one iteration apart at rtol 1e-12
    for q1, q2 in zip(s1.convergence, s2.convergence):
        assert abs(q1.iterations - q2.iterations) <= 1
        assert q1.residual_norm <= 1e-12 * q1.rhs_norm
    assert np.linalg.norm(s1.value - s2.value) <= 1e-9 * np.linalg.norm(s2.value)
