"""The matrix-free operator (I - T C) x in its three device forms against the oracle.

lmax 2..5 run the product form (harmonic tables of a chunk of sources times the coefficient
block, then the plan's term lists once per destination; TCU_APPLY=fly keeps it for several
columns too); lmax 1 and >= 6, or TCU_APPLY=terms, run the per-pair term sums. The stored form
(the default for several columns and inside GMRES, forced by TCU_APPLY=stored) builds the
tables of all pairs once and applies the FP64 tensor-core product over them. 37 spheres make the destination groups and the source chunks of the
product form ragged; three right-hand sides exercise the column grid. Bound: relative 1e-13 in
the 2-norm against the oracle's FP64 operator (cluster/iterative.rs apply path).
"""
import numpy as np
import pytest

import oracle
from treams_b200 import workloads

pytestmark = pytest.mark.gpu


def _rel(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


@pytest.mark.parametrize("lmax", [1, 2, 3, 4, 5, 6])
@pytest.mark.parametrize("form", ["default", "fly", "terms", "stored"])
def test_operator_forms_match_the_oracle(ctx, lmax, form, monkeypatch):
    import treams_b200 as t
    if form == "default":
        monkeypatch.delenv("TCU_APPLY", raising=False)
    else:
        monkeypatch.setenv("TCU_APPLY", form)
    w = workloads.learned_cluster(seed=90 + lmax, count=37)
    n = w.radii.size * 2 * lmax * (lmax + 2)
    rng = np.random.default_rng(lmax)
    x = rng.standard_normal((n, 3)) + 1j * rng.standard_normal((n, 3))
    yg = t.cluster_apply(lmax, w.k0, w.radii, w.eps, w.positions, x, ctx=ctx)
    yo = oracle.iterative_apply(lmax, w.k0, w.radii, w.eps, w.positions, x)
    assert _rel(yg, yo) <= 1e-13


def test_product_and_term_forms_agree_at_4096_spheres(ctx, monkeypatch):
    # the 4096-sphere GMRES workload (lmax 3, n = 122,880): both device forms, one column
    import treams_b200 as t
    w = workloads.learned_cluster()
    x = np.random.default_rng(11).standard_normal(w.n) + 0j
    monkeypatch.delenv("TCU_APPLY", raising=False)
    yp = t.cluster_apply(w.lmax, w.k0, w.radii, w.eps, w.positions, x, ctx=ctx)
    monkeypatch.setenv("TCU_APPLY", "terms")
    yt = t.cluster_apply(w.lmax, w.k0, w.radii, w.eps, w.positions, x, ctx=ctx)
    assert _rel(yp, yt) <= 1e-13


def test_stored_and_product_forms_agree_at_4096_spheres(ctx, monkeypatch):
    # the stored tables of the 4096-sphere workload take 14 GB of HBM
    import treams_b200 as t
    w = workloads.learned_cluster()
    x = np.random.default_rng(12).standard_normal((w.n, 2)) + 0j
    monkeypatch.setenv("TCU_APPLY", "fly")
    yp = t.cluster_apply(w.lmax, w.k0, w.radii, w.eps, w.positions, x, ctx=ctx)
    monkeypatch.delenv("TCU_APPLY", raising=False)
    ys = t.cluster_apply(w.lmax, w.k0, w.radii, w.eps, w.positions, x, ctx=ctx)
    assert _rel(ys, yp) <= 1e-13


@pytest.mark.parametrize("lmax", [2, 3, 4, 5])
def test_gmres_with_stored_tables_matches_the_on_the_fly_product(ctx, lmax, monkeypatch):
    # GMRES builds the tables once per solve (default) or applies the product form every time
    import treams_b200 as t
    w = workloads.learned_cluster(seed=120 + lmax, count=150)
    c = t.SphereCluster(lmax, w.k0, w.radii, w.eps, w.positions, ctx=ctx)
    pw = t.plane_wave_expansion(lmax, w.positions, w.kvecs, w.pols, ctx=ctx)[:, 0]
    rng = np.random.default_rng(lmax)
    B = np.column_stack([pw, rng.standard_normal(pw.size) + 1j * rng.standard_normal(pw.size)])
    monkeypatch.delenv("TCU_APPLY", raising=False)
    s1 = c.solve(B, rtol=1e-12, restart=40, max_iterations=400)
    monkeypatch.setenv("TCU_APPLY", "fly")
    s2 = c.solve(B, rtol=1e-12, restart=40, max_iterations=400)
    assert [q.iterations for q in s1.convergence] == [q.iterations for q in s2.convergence]
    assert _rel(s1.value, s2.value) <= 1e-11


@pytest.mark.parametrize("lmax", [2, 3, 4, 5])
@pytest.mark.parametrize("pipe", ["cpasync", "tma"])
def test_stored_product_pipelines_match_the_oracle(ctx, lmax, pipe, monkeypatch):
    # both ways of streaming the stored tables into shared memory, forced at every lmax
    import treams_b200 as t
    monkeypatch.setenv("TCU_APPLY", "stored")
    monkeypatch.setenv("TCU_STORED_PIPE", pipe)
    w = workloads.learned_cluster(seed=140 + lmax, count=53)
    n = w.radii.size * 2 * lmax * (lmax + 2)
    rng = np.random.default_rng(lmax + 7)
    x = rng.standard_normal((n, 2)) + 1j * rng.standard_normal((n, 2))
    yg = t.cluster_apply(lmax, w.k0, w.radii, w.eps, w.positions, x, ctx=ctx)
    yo = oracle.iterative_apply(lmax, w.k0, w.radii, w.eps, w.positions, x)
    assert _rel(yg, yo) <= 1e-13
