"""Batched heterogeneous cluster solves against the oracle's dense FP64 solves.

Each cluster of the batch is checked on its own (relative error <= 1e-10, the tolerance of the
single-cluster tests), at lmax 3 to 6 (the degrees of the 256-cluster sweep); the batch orders
clusters by size and releases each operator before the next, so the results must equal those
of separate calls.
"""
import numpy as np
import pytest

import oracle
import treams_b200 as t
from treams_b200 import workloads

pytestmark = pytest.mark.gpu


def _small_batch():
    out = []
    for c, count in zip(range(4), (10, 24, 6, 16)):
        w = workloads.batch_cluster(c)
        # keep the test small: the first `count` spheres of the cluster, lmax capped at 4
        lmax = min(w.lmax, 4)
        out.append((lmax, w.k0, w.radii[:count], w.eps[:count], w.positions[:count]))
    # the sweep's highest degrees: first clusters of the sweep drawn with lmax 5 and 6, at
    # their own lmax (n = 700 and 768 for 10 and 8 spheres)
    for lmax, count in ((5, 10), (6, 8)):
        c = next(c for c in range(256) if workloads.batch_cluster(c).lmax == lmax)
        w = workloads.batch_cluster(c)
        out.append((lmax, w.k0, w.radii[:count], w.eps[:count], w.positions[:count]))
    return out


@pytest.mark.parametrize("precision", ["fp64", "mixed", "auto"])
def test_batch_matches_separate_oracle_solves(ctx, precision):
    batch, refs = [], []
    for lmax, k0, r, e, x in _small_batch():
        kv = np.array([[0, 0, k0]], complex)
        B = oracle.plane_wave_expansion(lmax, x, kv, np.array([1], np.int32))
        A, tb = oracle.cluster_operator(lmax, k0, r, e, x)
        refs.append(oracle.dense_solve(lmax, A, tb, B))
        batch.append((lmax, k0, r, e, x, B))
    X, certs, order = t.batch_solve(batch, precision, ctx=ctx)
    sizes = [b[2].size * 2 * b[0] * (b[0] + 2) for b in batch]
    assert [sizes[i] for i in order] == sorted(sizes, reverse=True)
    for Xi, Ri, ci in zip(X, refs, certs):
        assert np.linalg.norm(Xi - Ri) <= 1e-10 * np.linalg.norm(Ri)
        assert ci[0].residual_norm <= 1e-12 * ci[0].rhs_norm


def test_batch_reports_the_failing_cluster(ctx):
    lmax, k0, r, e, x = _small_batch()[0]
    bad = x.copy()
    bad[1] = bad[0]  # two spheres at one place
    B = np.ones((r.size * 2 * lmax * (lmax + 2), 1), complex)
    with pytest.raises(ValueError, match="cluster 1"):
        t.batch_solve([(lmax, k0, r, e, x, B), (lmax, k0, r, e, bad, B)], "fp64", ctx=ctx)


def test_stalled_mixed_refinement_falls_back_to_a_second_factor():
    # Cluster 18 of the sweep (28 spheres, lmax 6, k0 d down to 0.21): the mixed factor refines
    # to 1e-13 (with FP16 pieces, opt-in, after one step to TF32 pieces). Demanding a residual
    # no refinement reaches (1e-300) then exercises the last level of the chain, FP64.
    ctx = t.Context(0)
    try:
        w = workloads.batch_cluster(18)
        B = t.plane_wave_expansion(w.lmax, w.positions, w.kvecs, w.pols, ctx=ctx)
        ref = t.sphere_cluster_factor(w.lmax, w.k0, w.radii, w.eps, w.positions, "fp64", ctx=ctx)
        X0, _ = ref.solve(B)
        f = t.sphere_cluster_factor(w.lmax, w.k0, w.radii, w.eps, w.positions, "mixed", ctx=ctx)
        X1, c1 = f.solve(B)
        first = ctx.fallbacks
        assert first <= 1  # at most the step to TF32 pieces
        assert c1[0].residual_norm <= 1e-13 * c1[0].rhs_norm
        assert np.linalg.norm(X1 - X0) <= 1e-10 * np.linalg.norm(X0)
        ctx.set_refinement(1e-13, 1e-300)
        X, certs = f.solve(B)
        assert ctx.fallbacks > first
        assert certs[0].residual_norm <= 1e-12 * certs[0].rhs_norm
        assert np.linalg.norm(X - X0) <= 1e-10 * np.linalg.norm(X0)
        n2 = ctx.fallbacks
        X2, _ = f.solve(B)  # the second factors are kept
        assert ctx.fallbacks > n2 and np.array_equal(X2, X)
    finally:
        ctx.close()


def test_fp16_pieces_opt_in_reaches_the_fp64_target():
    # TCU_SPLIT=f16 (read once per process, so in a child) switches the 3-pass split to
    # row-scaled FP16 pieces; the solve must still reach the FP64 target, directly or through
    # the fallback chain, and agree with the FP64 factor.
    import os
    import subprocess
    import sys

    from conftest import ROOT

    code = """
import numpy as np, treams_b200 as t
from treams_b200 import workloads
w = workloads.precision_cluster(count=64)
ctx = t.Context(0)
B = t.plane_wave_expansion(w.lmax, w.positions, w.kvecs, w.pols, ctx=ctx)
X0, _ = t.sphere_cluster_factor(w.lmax, w.k0, w.radii, w.eps, w.positions, 'fp64', ctx=ctx).solve(B)
X, c = t.sphere_cluster_factor(w.lmax, w.k0, w.radii, w.eps, w.positions, 'mixed', ctx=ctx).solve(B)
print(max(x.residual_norm / x.rhs_norm for x in c), np.linalg.norm(X - X0) / np.linalg.norm(X0), ctx.fallbacks)
ctx.close()
"""
    env = dict(os.environ, TCU_SPLIT="f16", PYTHONPATH=f"{ROOT}:{ROOT / 'treams-rs_b200'}")
    out = subprocess.run([sys.executable, "-c", code], env=env, capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stderr[-2000:]
    res, err, fallbacks = out.stdout.split()
    assert float(res) <= 1e-12 and float(err) <= 1e-10


def test_autotuned_crossover_drives_auto_precision():
    ctx = t.Context(0)
    try:
        tuned = ctx.autotune()
        assert tuned["crossover"] in tuned["sizes"] or tuned["crossover"] > max(tuned["sizes"])
        assert all(v > 0 for v in tuned["ms_fp64"] + tuned["ms_mixed"])
        batch, refs = [], []
        for lmax, k0, r, e, x in _small_batch()[:3]:
            kv = np.array([[0, 0, k0]], complex)
            B = oracle.plane_wave_expansion(lmax, x, kv, np.array([1], np.int32))
            A, tb = oracle.cluster_operator(lmax, k0, r, e, x)
            refs.append(oracle.dense_solve(lmax, A, tb, B))
            batch.append((lmax, k0, r, e, x, B))
        X, certs, _ = t.batch_solve(batch, "auto", ctx=ctx)
        for Xi, Ri in zip(X, refs):
            assert np.linalg.norm(Xi - Ri) <= 1e-10 * np.linalg.norm(Ri)
    finally:
        ctx.close()


def test_worker_threads_give_the_sequential_results(ctx, monkeypatch):
    # 12 clusters of the sweep (whole clusters: n up to ~20,000, mixed and FP64 by the crossover)
    # solved by 4 host workers with a stream each and by one: the same factors and refinements,
    # so the same solutions and certificates
    batch = []
    for c in range(12):
        w = workloads.batch_cluster(c)
        B = t.plane_wave_expansion(w.lmax, w.positions, w.kvecs, w.pols, ctx=ctx)
        batch.append((w.lmax, w.k0, w.radii, w.eps, w.positions, B))
    monkeypatch.setenv("TCU_BATCH_WORKERS", "4")
    X4, c4, o4 = t.batch_solve(batch, "auto", ctx=ctx)
    monkeypatch.setenv("TCU_BATCH_WORKERS", "1")
    X1, c1, o1 = t.batch_solve(batch, "auto", ctx=ctx)
    assert o4 == o1
    for a, b, ca, cb in zip(X4, X1, c4, c1):
        assert np.linalg.norm(a - b) <= 1e-13 * np.linalg.norm(b)
        assert ca[0].residual_norm <= 1e-12 * ca[0].rhs_norm
