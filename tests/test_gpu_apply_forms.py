"""The matrix-free operator (I - T C) x in its two device forms against the oracle.

lmax 2..5 run the product form (harmonic tables of a chunk of sources times the coefficient
block, then the plan's term lists once per destination); lmax 1 and >= 6, or TCU_APPLY=terms,
run the per-pair term sums. 37 spheres make the destination groups and the source chunks of the
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
@pytest.mark.parametrize("form", ["product", "terms"])
def test_operator_forms_match_the_oracle(ctx, lmax, form, monkeypatch):
    import treams_b200 as t
    if form == "terms":
        monkeypatch.setenv("TCU_APPLY", "terms")
    else:
        monkeypatch.delenv("TCU_APPLY", raising=False)
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
