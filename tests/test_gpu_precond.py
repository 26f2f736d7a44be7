"""Preconditioned matrix-free GMRES on the GPU and the learned preconditioner's network.

The preconditioners have no reference counterpart (the reference's iterative solver is
unpreconditioned), so the checks are:
(1) the training loss of the graph network and its gradient from the device's forward and
    backward kernels against the oracle's restatement (oracle.gnn_loss: the same graph,
    features, network, near-field blocks and dense FP64 operator): the loss to 1e-10 relative,
    the gradient against central differences of the oracle's loss (relative 1e-6 per checked
    weight and along a random direction);
(2) preconditioned solves against the oracle's dense FP64 solve, the FP64 residual
    certificate as the criterion (relative error 1e-8 at rtol 1e-10);
(3) what each level gains: the two-level methods need fewer iterations than block Jacobi, and
    the trained network no more than the two-level method without it.
"""
import numpy as np
import pytest

import oracle
import treams_b200 as t
from treams_b200 import workloads

pytestmark = pytest.mark.gpu


def _cluster(count, seed):
    return workloads.learned_cluster(seed=seed, count=count)


def test_network_loss_and_gradient_match_the_oracle(ctx):
    from treams_b200.train_precond import init_weights
    w = _cluster(20, 77)
    rng = np.random.default_rng(5)
    V = rng.standard_normal((w.n, 2)) + 1j * rng.standard_normal((w.n, 2))
    prob = t.LearnedProblem(w.lmax, w.k0, w.radii, w.eps, w.positions, V, ctx=ctx)
    try:
        R1 = prob.probes()
        assert np.allclose(np.linalg.norm(R1, axis=0), 1.0, rtol=1e-12)
        W = init_weights(3, seed=3)
        W += 0.05 * rng.standard_normal(W.size)  # nonzero output layer: Theta != 1
        loss, grad = prob.loss_grad(W)
        A, tb = oracle.cluster_operator(w.lmax, w.k0, w.radii, w.eps, w.positions)
        f = lambda x: oracle.gnn_loss(w.lmax, w.k0, w.radii, w.eps, w.positions, R1, x, A=A, tb=tb)  # noqa: E731
        lo = f(W)
        assert abs(loss - lo) <= 1e-10 * abs(lo), (loss, lo)
        h = 1e-5
        lay, total = oracle.gnn_layout(3)
        picks = [lay[name][0] + int(rng.integers(0, np.prod(lay[name][1]))) for name in lay for _ in range(2)]
        for i in picks:
            e = np.zeros_like(W)
            e[i] = h
            fd = (f(W + e) - f(W - e)) / (2 * h)
            assert abs(grad[i] - fd) <= 1e-6 * max(abs(fd), 1e-3 * np.abs(grad).max()), (i, grad[i], fd)
        d = rng.standard_normal(W.size)
        d /= np.linalg.norm(d)
        fd = (f(W + h * d) - f(W - h * d)) / (2 * h)
        assert abs(grad @ d - fd) <= 1e-6 * abs(fd)
    finally:
        prob.close()


@pytest.mark.parametrize("kind", ["block_jacobi", "two_level", "learned"])
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


def test_two_level_and_learned_gains_on_a_held_out_cluster(ctx):
    # 512 spheres of the 4096-sphere workload's distribution (seed outside the training set):
    # iterations to 1e-8 with GMRES(50)
    w = _cluster(512, 4242)
    c = t.SphereCluster(w.lmax, w.k0, w.radii, w.eps, w.positions, ctx=ctx)
    B = t.plane_wave_expansion(w.lmax, w.positions, w.kvecs, w.pols, ctx=ctx)[:, 0]
    its = {}
    for kind in ("none", "block_jacobi", "two_level", "learned"):
        sol = c.solve(B, rtol=1e-8, restart=50, max_iterations=400, preconditioner=kind)
        cert = sol.convergence[0]
        assert cert.residual_norm <= 1e-8 * cert.rhs_norm
        its[kind] = cert.iterations
    assert its["two_level"] * 2 <= its["block_jacobi"], its
    assert its["learned"] <= its["two_level"], its


def test_block_jacobi_with_one_sphere_blocks_is_the_identity(ctx):
    # at lmax 5 a block holds one sphere (70 modes), whose own system is I: plain GMRES
    w = workloads.small_cluster()
    c = t.SphereCluster(5, w.k0, w.radii, w.eps, w.positions, ctx=ctx)
    b = np.random.default_rng(3).standard_normal(c.dimension) + 0j
    p = c.solve(b, rtol=1e-10)
    q = c.solve(b, rtol=1e-10, preconditioner="block_jacobi")
    assert q.convergence[0].iterations == p.convergence[0].iterations
    assert np.linalg.norm(q.value - p.value) <= 1e-9 * np.linalg.norm(p.value)


def test_two_level_with_the_iterative_dipole_solve(ctx):
    # 1200 spheres: 7200 dipole modes, above the size where the dipole system is factored, so
    # the two-level preconditioner solves it by the inner GMRES (a varying preconditioner the
    # flexible outer GMRES accepts). The FP64 residual certificate is the criterion; the solution
    # agrees with block Jacobi's and keeps the two-level iteration gain.
    w = _cluster(1200, 4343)
    c = t.SphereCluster(w.lmax, w.k0, w.radii, w.eps, w.positions, ctx=ctx)
    B = t.plane_wave_expansion(w.lmax, w.positions, w.kvecs, w.pols, ctx=ctx)[:, 0]
    sols = {}
    for kind in ("block_jacobi", "two_level"):
        sol = c.solve(B, rtol=1e-10, restart=50, max_iterations=400, preconditioner=kind)
        cert = sol.convergence[0]
        assert cert.residual_norm <= 1e-10 * cert.rhs_norm
        sols[kind] = sol
    x0 = sols["block_jacobi"].value
    assert np.linalg.norm(sols["two_level"].value - x0) <= 1e-8 * np.linalg.norm(x0)
    its = {k: s.convergence[0].iterations for k, s in sols.items()}
    assert its["two_level"] * 2 <= its["block_jacobi"], its
