"""The headline workload itself against the oracle: the 512-sphere lmax-4 cluster (seed 1002,
n = 24,576, three plane waves) solved on the GPU in mixed precision and in FP64, compared with
the oracle's FP64 assembly of I - T C plus LAPACK zgetrf/zgetrs on the host cores.

Tolerances: relative error <= 1e-10 in the scattered coefficients of each
column and in sigma_sca and sigma_ext. The host side needs about 10 GB of memory and a minute
or two of LAPACK time.
"""
import numpy as np
import pytest

import oracle
from treams_b200 import workloads

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def headline():
    w = workloads.precision_cluster()
    B = oracle.plane_wave_expansion(w.lmax, w.positions, w.kvecs, w.pols)
    X = oracle.lapack_cluster_solve(w.lmax, w.k0, w.radii, w.eps, w.positions, B)
    sections = [oracle.cross_sections(w.lmax, w.k0, w.positions, X[:, c], B[:, c]) for c in range(B.shape[1])]
    return w, B, X, sections


@pytest.mark.parametrize("precision", ["mixed", "fp64"])
def test_headline_cluster_matches_the_oracle(ctx, headline, precision):
    import treams_b200 as t
    w, B, Xo, sections = headline
    f = t.sphere_cluster_factor(w.lmax, w.k0, w.radii, w.eps, w.positions, precision, ctx=ctx)
    try:
        X, certs = f.solve(B)
    finally:
        f.close()
    for c in range(B.shape[1]):
        err = np.linalg.norm(X[:, c] - Xo[:, c]) / np.linalg.norm(Xo[:, c])
        assert err <= 1e-10, (precision, c, err)
        assert certs[c].residual_norm <= 1e-12 * certs[c].rhs_norm
    sca, ext = t.cross_sections(w.lmax, w.k0, w.positions, X, B, ctx=ctx)
    for c in range(B.shape[1]):
        so, eo = sections[c]
        assert abs(sca[c] - so) <= 1e-10 * abs(so), (c, sca[c], so)
        assert abs(ext[c] - eo) <= 1e-10 * abs(eo), (c, ext[c], eo)
