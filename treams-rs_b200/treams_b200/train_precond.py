"""Fit the layer weights of the learned GMRES preconditioner and write them into the library.

The preconditioner is M = sum_k alpha_k (D N)^k D (block-Jacobi inverse D, near-field couplings
N between blocks; csrc/precond.cu). Its loss on a probe vector v is ||v - A M v||^2 with
A = I - T C, which is quadratic in alpha: summed over probe vectors it equals
const - 2 Re(alpha^H b) + alpha^H G alpha with the statistics (G, b) that the GPU returns
(tcu_learned_precond_gram; its gradient 2 (G alpha - b) is checked against the CPU oracle in
the GPU tests). Training minimises the loss over training clusters (seeds 2000 + i,
N ~ U{64..1024}, the 4096-sphere workload's material and packing), each probe normalised to
unit norm, with a small ridge term; the minimiser solves (G + lambda I) alpha = b.

Run on a GPU:  python -m treams_b200.train_precond [--clusters 12] [--layers 6] [--reach 6] --write
It rewrites treams-rs_b200/csrc/learned_coefficients.inc; rebuild the library afterwards.
"""
from __future__ import annotations

import argparse
import pathlib

import numpy as np

from . import _lib, workloads

INC = pathlib.Path(__file__).resolve().parent.parent / "csrc" / "learned_coefficients.inc"


def statistics(i: int, layers: int, nrandom: int, ctx) -> tuple[np.ndarray, np.ndarray, float]:
    w = workloads.training_cluster(i)
    rng = np.random.default_rng(7000 + i)
    probes = [rng.standard_normal(w.n) + 1j * rng.standard_normal(w.n) for _ in range(nrandom)]
    # the incident field T b of a plane wave along +z, the right-hand side GMRES sees
    B = _lib.plane_wave_expansion(w.lmax, w.positions, w.kvecs, w.pols, ctx=ctx)[:, 0]
    T = _lib.mie_blocks(w.lmax, w.k0, w.radii, w.eps, ctx=ctx)
    tb = np.empty_like(B)
    M = 2 * w.lmax * (w.lmax + 2)
    for s in range(w.radii.size):
        for lm in range(M // 2):
            l = int(np.sqrt(lm + 1))
            t4 = T[s, l - 1]
            x = B[s * M + 2 * lm: s * M + 2 * lm + 2]
            tb[s * M + 2 * lm: s * M + 2 * lm + 2] = t4 @ x
    probes.append(tb)
    V = np.stack([p / np.linalg.norm(p) for p in probes], axis=1)
    G, b = _lib.learned_precond_gram(w.lmax, w.k0, w.radii, w.eps, w.positions, layers, V, ctx=ctx)
    return G, b, float(V.shape[1])


def fit(clusters: int, layers: int, nrandom: int = 3, ridge: float = 1e-8, ctx=None):
    ctx = ctx or _lib.default_context()
    K1 = layers + 1
    G = np.zeros((K1, K1), complex)
    b = np.zeros(K1, complex)
    total = 0.0
    for i in range(clusters):
        g, r, nv = statistics(i, layers, nrandom, ctx)
        G += g
        b += r
        total += nv
    scale = np.trace(G).real / K1
    alpha = np.linalg.solve(G + ridge * scale * np.eye(K1), b)
    loss = lambda a: (total - 2 * np.real(np.vdot(a, b)) + np.real(np.vdot(a, G @ a))) / total
    e0 = np.zeros(K1, complex)
    e0[0] = 1.0
    return alpha, {"loss_fit": loss(alpha), "loss_block_jacobi": loss(e0), "loss_relaxation": loss(np.ones(K1)),
                   "probes": total}


def write_inc(alpha_by_lmax: dict[int, np.ndarray], layers: int, reach: float, note: str) -> None:
    lines = [
        "// Layer weights alpha_k of the learned preconditioner per lmax (generated by",
        "// treams-rs_b200/treams_b200/train_precond.py from least-squares fits on training clusters;",
        "// lmax without a fit uses alpha_k = 1, i.e. plain block-Jacobi relaxation sweeps).",
        f"// {note}",
        f"constexpr int LEARNED_LAYERS = {layers};",
        f"constexpr double LEARNED_REACH = {float(reach)!r};",
        "inline std::complex<double> learned_alpha(int lmax, int k) {",
    ]
    for L, a in sorted(alpha_by_lmax.items()):
        vals = ", ".join(f"{{{float(z.real)!r}, {float(z.imag)!r}}}" for z in a)
        lines.append(f"    static const double a{L}[][2] = {{{vals}}};")
        lines.append(f"    if (lmax == {L} && k >= 0 && k < {len(a)}) return {{a{L}[k][0], a{L}[k][1]}};")
    lines += ["    (void)lmax;", "    (void)k;", "    return {1.0, 0.0};", "}", ""]
    INC.write_text("\n".join(lines))


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--clusters", type=int, default=12)
    ap.add_argument("--layers", type=int, default=6)
    ap.add_argument("--reach", type=float, default=6.0, help="near-field reach in sphere diameters")
    ap.add_argument("--write", action="store_true", help="rewrite csrc/learned_coefficients.inc")
    args = ap.parse_args()
    ctx = _lib.default_context()
    ctx.set_learned_preconditioner(args.reach, layers=args.layers)
    alpha, info = fit(args.clusters, args.layers, ctx=ctx)
    print({"alpha": [complex(a) for a in alpha], **info})
    if args.write:
        write_inc({3: alpha}, args.layers, args.reach,
                  f"fit on {args.clusters} training clusters at reach {args.reach:g} diameters: mean probe loss "
                  f"{info['loss_fit']:.4g} (relaxation {info['loss_relaxation']:.4g}, block Jacobi "
                  f"{info['loss_block_jacobi']:.4g})")


if __name__ == "__main__":
    main()
