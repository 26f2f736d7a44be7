"""GPU 2D lattice sums and the batched periodic-array solve against the binary128 oracle.

Tolerances: lattice sums to 1e-11 * max(|D|, 1) over the whole table (the reference checks its
own sums to 2.5e-13 * max(|S|, 1) of 30-digit values; the device path works in FP64 with
series and continued fractions whose rounding we bound at ~1e-13 per term, and the largest
tables reach |D| ~ 1e7 at l = 12); array solves to 1e-10 * max(|X|).
"""
import math

import numpy as np
import pytest

import oracle
from conftest import read_table
from treams_b200 import lattice as tl
from treams_b200 import workloads

pytestmark = pytest.mark.gpu


def _check_table(D, lsum, k, lat, kps, eta=0.0, tol=1e-11):
    for i, kp in enumerate(kps):
        ref = oracle.lsumsw2d_table(lsum, k, lat, kp, eta=eta)
        scale = max(1.0, np.max(np.abs(ref)))
        err = np.max(np.abs(D[i] - ref)) / scale
        assert err <= tol, (i, kp, err)


@pytest.mark.parametrize("draw", [0, 3])
def test_lattice_sums_periodic_workload(ctx, draw):
    # the 4096-Bloch-vector square-lattice workload (k0 = 4, degrees <= 12), checked on a subset
    w = workloads.periodic_array(draw=draw)
    kps = w.kpars[:24]
    D = tl.lsumsw2d_batch(12, w.k0, w.lattice, kps, ctx=ctx)
    assert D.shape == (24, 169)
    _check_table(D[::4], 12, w.k0, w.lattice, kps[::4])


def test_lattice_sums_hexagonal_and_explicit_split(ctx):
    lat = np.array([[1.0, 0.0], [0.5, math.sqrt(3) / 2]])
    kps = np.array([[0.3, -0.2], [1.1, 0.4], [-2.0, 0.7]])
    for eta in (0.0, 0.6):
        D = tl.lsumsw2d_batch(9, 2.7, lat, kps, eta=eta, ctx=ctx)
        _check_table(D, 9, 2.7, lat, kps, eta=eta)


def test_lattice_sums_oblique_large_kl(ctx):
    # |k L| > 8 selects the larger automatic split (cell.rs:164-175)
    lat = np.array([[1.4, 0.0], [0.5, 1.6]])
    kps = np.array([[0.4, -0.7], [0.0, 0.0]])
    D = tl.lsumsw2d_batch(6, 7.3, lat, kps, ctx=ctx)
    _check_table(D, 6, 7.3, lat, kps)


def test_lattice_sums_are_bloch_periodic_on_device(ctx):
    w = workloads.periodic_array()
    g = 2 * math.pi / w.period
    kp = np.array([w.kpars[7], w.kpars[7] + np.array([-g, g])])
    D = tl.lsumsw2d_batch(12, w.k0, w.lattice, kp, ctx=ctx)
    assert np.max(np.abs(D[1] - D[0])) <= 1e-11 * max(1.0, np.max(np.abs(D[0])))


def test_lattice_sum_at_a_diffraction_threshold_is_rejected(ctx):
    # |kpar + G| = k for G = 0 (lattice/mod.rs failure table)
    with pytest.raises(ValueError, match="diffraction threshold"):
        tl.lsumsw2d_batch(4, 2.0, np.eye(2), np.array([[2.0, 0.0]]), ctx=ctx)


def test_lattice_sum_invalid_inputs(ctx):
    with pytest.raises(ValueError):
        tl.lsumsw2d_batch(4, -1.0, np.eye(2), np.array([[0.1, 0.0]]), ctx=ctx)
    with pytest.raises(ValueError):
        tl.lsumsw2d_batch(4, 1.0, np.array([[1.0, 0.0], [2.0, 0.0]]), np.array([[0.1, 0.0]]), ctx=ctx)
    with pytest.raises(ValueError):
        tl.lsumsw2d_batch(15, 1.0, np.eye(2), np.array([[0.1, 0.0]]), ctx=ctx)
    with pytest.raises(ValueError, match="split"):
        tl.lsumsw2d_batch(4, 1.0, np.eye(2), np.array([[0.1, 0.0]]), eta=0.1, ctx=ctx)


@pytest.mark.parametrize("draw", [0, 5])
def test_array_solve_matches_oracle(ctx, draw):
    w = workloads.periodic_array(draw=draw)
    kps = w.kpars[:6]
    X = tl.array_solve_batch(w.lmax, w.k0, w.radius, w.eps, w.lattice, kps, ctx=ctx)
    assert X.shape == (6, 96, 96)
    for i in (0, 3, 5):
        ref = oracle.array_solve(w.lmax, w.k0, w.radius, w.eps, w.lattice, kps[i])
        err = np.max(np.abs(X[i] - ref)) / np.max(np.abs(ref))
        assert err <= 1e-10, (i, err)


def test_array_solve_small_lmax_lossy(ctx):
    lat = np.array([[0.9, 0.0], [0.3, 0.8]])
    kps = np.array([[0.5, 0.1], [-1.2, 2.0]])
    X = tl.array_solve_batch(3, 2.5, 0.25, 3.0 + 0.4j, lat, kps, ctx=ctx)
    for i in range(2):
        ref = oracle.array_solve(3, 2.5, 0.25, 3.0 + 0.4j, lat, kps[i])
        assert np.max(np.abs(X[i] - ref)) <= 1e-10 * np.max(np.abs(ref))


@pytest.mark.parametrize("lmax", [1, 2, 4, 5])
def test_array_solve_every_operator_size(ctx, lmax):
    # M = 6, 16, 48, 70: one to nine warps of eight rows, partial row blocks (M = 6, 70) and
    # partial column tiles (M = 16, 70) of the register-resident Gauss-Jordan kernel
    lat = np.array([[0.9, 0.0], [0.3, 0.8]])
    kps = np.array([[0.5, 0.1], [-1.2, 2.0], [0.0, 0.0]])
    X = tl.array_solve_batch(lmax, 2.5, 0.25, 3.0 + 0.4j, lat, kps, ctx=ctx)
    for i in range(len(kps)):
        ref = oracle.array_solve(lmax, 2.5, 0.25, 3.0 + 0.4j, lat, kps[i])
        assert np.max(np.abs(X[i] - ref)) <= 1e-10 * np.max(np.abs(ref)), (lmax, i)


def test_array_solve_rejects_touching_spheres(ctx):
    with pytest.raises(ValueError, match="overlap"):
        tl.array_solve_batch(2, 2.0, 0.6, 4.0, np.eye(2), np.array([[0.1, 0.2]]), ctx=ctx)


@pytest.mark.parametrize("shift", [(0.3, 0.1, 0.0), (-0.45, 0.2, 0.0), (2.4, -1.3, 0.0)])
def test_shifted_lattice_sums_match_oracle(ctx, shift):
    # in-plane shifts (two sphere positions of a multi-sphere cell); the last one lies outside
    # the cell and is reduced into it with the Bloch phase e^{-i kpar.R0} (lattice/ewald.rs:610-665)
    lat = np.array([[1.0, 0.0], [0.5, math.sqrt(3) / 2]])
    kps = np.array([[0.3, -0.2], [1.1, 0.4], [-2.0, 0.7]])
    D = tl.lsumsw2d_batch(8, 2.7, lat, kps, shift=shift, ctx=ctx)
    for i, kp in enumerate(kps):
        ref = oracle.lsumsw2d_table(8, 2.7, lat, kp, r=shift)
        assert np.max(np.abs(D[i] - ref)) <= 1e-11 * max(1.0, np.max(np.abs(ref))), (shift, i)


@pytest.mark.parametrize("shift", [(0.3, 0.1, 0.25), (-0.45, 0.2, -0.4), (0.0, 0.0, 0.15), (2.4, -1.3, 0.6)])
def test_off_plane_lattice_sums_match_oracle(ctx, shift):
    # shifts off the lattice plane (spheres of a cell at different heights): every order n <= l - |m|
    # of S_lmn and the t-series of F_(1/2-n)(v, t) (lattice/reciprocal.rs:22-60, lattice/reduced.rs:223)
    lat = np.array([[1.0, 0.0], [0.3, 0.9]])
    kps = np.array([[0.4, -0.7], [1.1, 0.4], [0.0, 0.0]])
    for eta in (0.0, 0.8):
        D = tl.lsumsw2d_batch(8, 2.7, lat, kps, eta=eta, shift=shift, ctx=ctx)
        for i, kp in enumerate(kps):
            ref = oracle.lsumsw2d_table(8, 2.7, lat, kp, r=shift, eta=eta)
            assert np.max(np.abs(D[i] - ref)) <= 1e-11 * max(1.0, np.max(np.abs(ref))), (shift, eta, i)


def test_off_plane_sums_do_not_depend_on_the_split(ctx):
    # the exact sum does not depend on eta (tests/lattice/test_lattice.py:300-308), off the plane too
    lat = np.array([[0.8, 0.0], [0.0, 0.8]])
    kps = np.array([[0.5, 0.2], [-1.0, 1.5]])
    d0 = tl.lsumsw2d_batch(10, 3.1, lat, kps, shift=(0.2, -0.1, 0.3), ctx=ctx)
    d1 = tl.lsumsw2d_batch(10, 3.1, lat, kps, eta=0.9, shift=(0.2, -0.1, 0.3), ctx=ctx)
    assert np.max(np.abs(d1 - d0)) <= 1e-11 * max(1.0, np.max(np.abs(d0)))


def test_shifted_sums_reject_shifts_far_off_the_plane(ctx):
    # off the plane the split is capped at |k r_z eta| <= 1 down to eta = 1/4 (1/(2 eta^2) <= 8);
    # beyond (k r_z eta)^2 = 16 the alternating t-series would lose FP64 accuracy: k r_z = 20 is rejected
    lat = np.eye(2)
    with pytest.raises(ValueError, match="off the lattice plane"):
        tl.lsumsw2d_batch(2, 2.0, lat, [[0.1, 0.2]], shift=(0.1, 0.0, 10.0), ctx=ctx)


@pytest.mark.parametrize("k", [2.7 + 0.4j, 1.5 + 0.05j])
@pytest.mark.parametrize("shift", [(0.0, 0.0, 0.0), (0.3, 0.1, 0.25), (0.2, -0.1, 0.0), (1.9, -2.2, -0.4)])
def test_complex_wavenumber_lattice_sums_match_oracle(ctx, k, shift):
    # a lossy embedding (lattice::sum at complex k, lattice/mod.rs:283): every diffraction order on
    # its outgoing sheet (lattice/sheets.rs); the device takes a real split, the oracle its automatic
    # complex one, and the sums do not depend on the split
    lat = np.array([[1.0, 0.0], [0.3, 0.9]])
    kps = np.array([[0.4, -0.7], [1.1, 0.4], [0.0, 0.0]])
    D = tl.lsumsw2d_batch(8, k, lat, kps, shift=shift, ctx=ctx)
    for i, kp in enumerate(kps):
        ref = oracle.lsumsw2d_table(8, k, lat, kp, r=shift)
        assert np.max(np.abs(D[i] - ref)) <= 1e-11 * max(1.0, np.max(np.abs(ref))), (k, shift, i)


def _golden_full_rows():
    rows = []
    for key, val in read_table("lattice_sums_2d.txt"):
        (_, l, m, dim, kr, ki, x, y, z, er, ei, a11, a12, a21, a22, b1, b2, part, jet, tol) = key
        k = complex(float(kr), float(ki))
        if part != "full" or float(ei) != 0.0 or not (k.real > 0 and 0 <= k.imag <= k.real / 2):
            continue
        rows.append(dict(l=int(l), m=int(m), k=k, r=[float(x), float(y), float(z)], eta=float(er),
                         lattice=[[float(a11), float(a12)], [float(a21), float(a22)]], kpar=[float(b1), float(b2)],
                         tol=float(tol), ref=complex(float(val[0]), float(val[1]))))
    return rows


def test_lattice_sums_match_reference_tables_on_the_device(ctx):
    # every 2D spherical full-sum row of the reference's high-precision table that the device path
    # takes (real split; Re k > 0, 0 <= Im k <= Re k / 2): complex k off the plane (image sums at 30
    # digits) and real k next to diffraction thresholds (spectral sums; q.q - k^2 from compensated
    # products with reciprocal vectors to twice FP64 precision), lattice/mod.rs:283.
    # Tolerance max(the row's own, 1e-12) * max(|S|, 1); the rows' own are 1e-14 to 1e-12.
    rows = _golden_full_rows()
    assert len(rows) >= 20
    for r in rows:
        D = tl.lsumsw2d_batch(r["l"], r["k"], r["lattice"], [r["kpar"]], eta=r["eta"], shift=r["r"], ctx=ctx)
        v = D[0, r["l"] * r["l"] + r["l"] + r["m"]]
        assert abs(v - r["ref"]) <= max(r["tol"], 1e-12) * max(1.0, abs(r["ref"])), (r, v)


def test_complex_wavenumber_sums_reject_strong_losses(ctx):
    with pytest.raises(ValueError, match="Im k"):
        tl.lsumsw2d_batch(2, 2.0 + 1.5j, np.eye(2), [[0.1, 0.2]], ctx=ctx)
