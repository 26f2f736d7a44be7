"""Failure detection on the GPU without a fault: a bounded device-side wait that runs out.

The LU panel's grid barrier runs with one arrival missing (a counter that nothing else
increments); its wait gives up after the limit, the host reads TCU_TIMEOUT, and the same
context then factors and solves a cluster correctly.
"""
import time

import numpy as np
import pytest

import oracle
from treams_b200 import workloads

pytestmark = pytest.mark.gpu


def test_bounded_wait_gives_up_and_context_stays_usable(ctx):
    import treams_b200 as t
    t0 = time.perf_counter()
    with pytest.raises(t.TreamsCudaError, match="gave up"):
        ctx.wait_selftest(0.05)
    elapsed = time.perf_counter() - t0
    assert 0.04 <= elapsed <= 3.0, elapsed
    # a second run in a row: the status word was cleared
    with pytest.raises(t.TreamsCudaError, match="gave up"):
        ctx.wait_selftest(0.01)
    w = workloads.small_cluster()
    A, tb = oracle.cluster_operator(w.lmax, w.k0, w.radii, w.eps, w.positions)
    B = oracle.plane_wave_expansion(w.lmax, w.positions, w.kvecs, w.pols)
    Xo = oracle.dense_solve(w.lmax, A, tb, B)
    f = t.sphere_cluster_factor(w.lmax, w.k0, w.radii, w.eps, w.positions, "mixed", ctx=ctx)
    try:
        X, certs = f.solve(B)
    finally:
        f.close()
    assert np.linalg.norm(X - Xo) <= 1e-10 * np.linalg.norm(Xo)
    assert certs[0].residual_norm <= 1e-12 * certs[0].rhs_norm


def test_selftest_rejects_bad_limit(ctx):
    with pytest.raises(ValueError):
        ctx.wait_selftest(float("nan"))
    with pytest.raises(ValueError):
        ctx.wait_selftest(-1.0)
