"""Preconditioned matrix-free GMRES on the GPU.

The preconditioners have no reference counterpart (parity unpinned: the reference's iterative
solver is unpreconditioned), so the checks are (1) the learned preconditioner's training
statistics against the CPU oracle's dense restatement of the same graph, blocks and layers (the
gradient 2 (G alpha - b) of the fit follows from them for every alpha), and (2) preconditioned
solves against the oracle's dense FP64 solve, with the FP64 residual certificate as the judge.
"""
import numpy as np
import pytest

import oracle
import treams_b200 as t
from treams_b200 import workloads

pytestmark = pytest.mark.gpu


def _cluster(count, seed):
    return workloads.learned_cluster(seed=seed, count=count)


@pytest.mark.parametrize("reach", [3.0, 6.0])
def test_learned_gram_matches_oracle(reach):
    ctx = t.Context(0)
    ctx.set_learned_preconditioner(reach, layers=3)
    w = _cluster(20, 77)
    rng = np.random.default_rng(5)
    n = w.n
    V = rng.standard_normal((n, 2)) + 1j * rng.standard_normal((n, 2))
    layers = 3
    G, b = t.learned_precond_gram(w.lmax, w.k0, w.radii, w.eps, w.positions, layers, V, ctx=ctx)
    Go, bo = oracle.learned_gram(w.lmax, w.k0, w.radii, w.eps, w.positions, layers, V, reach=reach)
    assert np.max(np.abs(G - Go)) <= 1e-10 * np.max(np.abs(Go))
    assert np.max(np.abs(b - bo)) <= 1e-10 * np.max(np.abs(bo))
    # gradient of the fit at a random alpha
    alpha = rng.standard_normal(layers + 1) + 1j * rng.standard_normal(layers + 1)
    g, go = 2 * (G @ alpha - b), 2 * (Go @ alpha - bo)
    assert np.max(np.abs(g - go)) <= 1e-10 * np.max(np.abs(go))
    ctx.close()


@pytest.mark.parametrize("kind", ["block_jacobi", "learned"])
def test_preconditioned_gmres_matches_dense_solve(ctx, kind):
    w = _cluster(48, 78)
    A, tb = oracle.cluster_operator(w.lmax, w.k0, w.radii, w.eps, w.positions)
    B = oracle.plane_wave_expansion(w.lmax, w.positions, w.kvecs, w.pols)
    X0 = oracle.dense_solve(w.lmax, A, tb, B)[:, 0]
    c = t.SphereCluster(w.lmax, w.k0, w.radii, w.eps, w.positions, ctx=ctx)
    plain = c.solve(B[:, 0], rtol=1e-10, restart=50, max_iterations=500)
    sol = c.solve(B[:, 0], rtol=1e-10, restart=50, max_iterations=500, preconditioner=kind)
    cert = sol.convergence[0]
    assert cert.residual_norm <= 1e-10 * cert.rhs_norm
    assert np.linalg.norm(sol.value - X0) <= 1e-8 * np.linalg.norm(X0)
    assert cert.iterations <= plain.convergence[0].iterations


def test_block_jacobi_with_one_sphere_blocks_is_the_identity(ctx):
    # at lmax 5 a block holds one sphere (70 modes), whose own system is I: plain GMRES
    w = workloads.small_cluster()
    c = t.SphereCluster(5, w.k0, w.radii, w.eps, w.positions, ctx=ctx)
    b = np.random.default_rng(3).standard_normal(c.dimension) + 0j
    p = c.solve(b, rtol=1e-10)
    q = c.solve(b, rtol=1e-10, preconditioner="block_jacobi")
    assert q.convergence[0].iterations == p.convergence[0].iterations
    assert np.linalg.norm(q.value - p.value) <= 1e-9 * np.linalg.norm(p.value)
