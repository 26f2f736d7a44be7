"""Seeded synthetic inputs of the five benchmark workloads (numpy PCG64).

Packing is random sequential addition: draw a centre uniformly in the box and a radius
from its distribution, reject the sphere if any gap to an accepted sphere is at or below
the required minimum, repeat. No public dataset is involved.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np


@dataclass
class Cluster:
    lmax: int
    k0: float
    radii: np.ndarray
    eps: np.ndarray
    positions: np.ndarray
    kvecs: np.ndarray  # (p, 3) complex wavevectors of the incident plane waves
    pols: np.ndarray   # (p,) helicity 0/1

    @property
    def n(self) -> int:
        return self.radii.size * 2 * self.lmax * (self.lmax + 2)


def _pack(rng, radii, side, gap):
    pos = np.zeros((len(radii), 3))
    for i, r in enumerate(radii):
        for _ in range(1_000_000):
            c = rng.uniform(0.0, side, 3)
            if i == 0:
                break
            d = np.linalg.norm(pos[:i] - c, axis=1) - radii[:i] - r
            if np.all(d > gap):
                break
        else:
            raise RuntimeError("packing failed")
        pos[i] = c
    return pos


def small_cluster(seed: int = 1001) -> Cluster:
    """8 spheres, r ~ U[0.2, 0.3], centres U([0, 2.5]^3), gaps > 0.05, eps 4+0.1i,
    k0 1.3, lmax 3 (n = 240); positive helicity plane wave along +z."""
    rng = np.random.default_rng(seed)
    radii, pos = [], []
    while len(radii) < 8:
        r = rng.uniform(0.2, 0.3)
        c = rng.uniform(0.0, 2.5, 3)
        if all(np.linalg.norm(c - p) - r - q > 0.05 for p, q in zip(pos, radii)):
            radii.append(r)
            pos.append(c)
    k0 = 1.3
    return Cluster(3, k0, np.array(radii), np.full(8, 4 + 0.1j), np.array(pos),
                   np.array([[0, 0, k0]], complex), np.array([1], np.int32))


def precision_cluster(seed: int = 1002, count: int = 512) -> Cluster:
    """512 spheres, r ~ U[0.15, 0.3], cubic box side (sum (4/3) pi r^3 / 0.15)^(1/3),
    strict separation, eps 2.25+0.01i, k0 2.0, lmax 4 (n = 24,576); three positive
    helicity plane waves along +z, +x and (sin 30, 0, cos 30)."""
    rng = np.random.default_rng(seed)
    radii = rng.uniform(0.15, 0.3, count)
    side = (np.sum(4.0 / 3.0 * np.pi * radii**3) / 0.15) ** (1.0 / 3.0)
    pos = _pack(rng, radii, side, 0.0)
    k0 = 2.0
    s, c = np.sin(np.pi / 6), np.cos(np.pi / 6)
    kv = np.array([[0, 0, k0], [k0, 0, 0], [k0 * s, 0, k0 * c]], complex)
    return Cluster(4, k0, radii, np.full(count, 2.25 + 0.01j), pos, kv, np.array([1, 1, 1], np.int32))


def learned_cluster(seed: int = 1004, count: int = 4096, fill: float = 0.2) -> Cluster:
    """4096 spheres r = 0.2 at 20% fill (box side ~ 8.82), eps 4+0.05i, k0 1.5, lmax 3
    (n = 122,880); positive helicity plane wave along +z."""
    rng = np.random.default_rng(seed)
    radii = np.full(count, 0.2)
    side = (count * 4.0 / 3.0 * np.pi * 0.2**3 / fill) ** (1.0 / 3.0)
    pos = _pack(rng, radii, side, 0.0)
    k0 = 1.5
    return Cluster(3, k0, radii, np.full(count, 4 + 0.05j), pos, np.array([[0, 0, k0]], complex),
                   np.array([1], np.int32))


def training_cluster(i: int) -> Cluster:
    """Training cluster i of the learned preconditioner: seed 2000 + i, N ~ U{64..1024}, otherwise
    the 4096-sphere workload's distribution (r = 0.2 at 20% fill, eps 4+0.05i, k0 1.5, lmax 3)."""
    rng = np.random.default_rng(2000 + i)
    count = int(rng.integers(64, 1025))
    return learned_cluster(seed=2000 + i, count=count)


def batch_cluster(c: int, seed: int = 1003) -> Cluster:
    """Cluster c of the 256-cluster sweep: N ~ U{16..256}, lmax ~ U{3..6}, k0 ~ U[0.5, 3],
    r ~ U[0.1, 0.3], Re eps ~ U[2, 6], Im eps ~ U[0, 0.2], box for 15% fill."""
    rng = np.random.default_rng(seed * 1000 + c)
    N = int(rng.integers(16, 257))
    lmax = int(rng.integers(3, 7))
    k0 = float(rng.uniform(0.5, 3.0))
    radii = rng.uniform(0.1, 0.3, N)
    eps = rng.uniform(2, 6, N) + 1j * rng.uniform(0, 0.2, N)
    side = (np.sum(4.0 / 3.0 * np.pi * radii**3) / 0.15) ** (1.0 / 3.0)
    pos = _pack(rng, radii, side, 0.0)
    return Cluster(lmax, k0, radii, eps, pos, np.array([[0, 0, k0]], complex), np.array([1], np.int32))


@dataclass
class PeriodicArray:
    lmax: int
    k0: float
    radius: float
    eps: complex
    period: float
    kpars: np.ndarray  # (nk, 2)

    @property
    def lattice(self) -> np.ndarray:
        return np.array([[self.period, 0.0], [0.0, self.period]])


def periodic_array(seed: int = 1005, nk: int = 4096, draw: int = 0) -> PeriodicArray:
    """Square lattice of period ~ U[0.5, 1.0] (draw-th draw), one sphere per cell r 0.2,
    eps 9, k0 4, lmax 6, nk Bloch vectors uniform in [-pi/a, pi/a)^2."""
    rng = np.random.default_rng(seed)
    periods = rng.uniform(0.5, 1.0, draw + 1)
    a = float(periods[draw])
    kp = rng.uniform(-np.pi / a, np.pi / a, (nk, 2))
    return PeriodicArray(6, 4.0, 0.2, 9.0 + 0j, a, kp)
