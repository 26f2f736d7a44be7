"""Train the graph network of the learned GMRES preconditioner on the GPU and write its weights
into the library.

The preconditioner (csrc/gnn.cu) is two-level: a coarse solve of the cluster's dipole system,
then the near field (pairs closer than 3 sphere diameters) with every (degree, degree) sub-block
of each translation block scaled by Theta_ij, which a small graph network predicts from node and
edge features. Training minimises the mean over coarse-corrected probe vectors r1 of
||r1 - A M_Theta r1||^2 (A = I - T C in FP64) over generated clusters (seeds 2000 + i,
N ~ U{64..1024}, the 4096-sphere workload's material and packing). The probes are the
right-hand sides the solver sees, T b for plane waves of several directions and helicities, and
random vectors. Loss and gradient come from the library's forward and backward kernels
(tcu_learned_problem_loss_grad); the optimiser (Adam) runs on the host over the few thousand
weights. Theta = 1 (all output weights zero) is the untrained two-level method, and training
starts there.

The probe loss is a one-step proxy: lowering it can still cost GMRES iterations (Theta can
absorb far-field coupling into the near-field blocks on average while spreading the spectrum).
So every `eval_every` steps the current weights run preconditioned GMRES(50) to 1e-8 on held-out
validation clusters (seeds 3000 + v, 512 spheres), and the weights kept are the ones with the
fewest total iterations (ties: the smaller summed relative residual), Theta = 1 included. When no
trained weights beat Theta = 1 the library keeps Theta = 1.

Run on a GPU:  python -m treams_b200.train_precond [--clusters 8] [--steps 300] --write
It rewrites treams-rs_b200/csrc/learned_weights.inc; rebuild the library afterwards.
"""
from __future__ import annotations

import argparse
import json
import pathlib
import time

import numpy as np

from . import _lib, workloads

INC = pathlib.Path(__file__).resolve().parent.parent / "csrc" / "learned_weights.inc"
H, NF, EF = 16, 6, 5


def init_weights(lmax: int, seed: int = 0) -> np.ndarray:
    """Random hidden layers (variance 1/fan-in), zero output layer: Theta = 1 at the start."""
    rng = np.random.default_rng(seed)
    nin, no = 2 * H + EF, 2 * lmax * lmax
    parts = [rng.standard_normal(H * NF) / np.sqrt(NF), np.zeros(H), rng.standard_normal(H * nin) / np.sqrt(nin),
             np.zeros(H), rng.standard_normal(H * nin) / np.sqrt(nin), np.zeros(H), np.zeros(no * H), np.zeros(no)]
    w = np.concatenate(parts)
    assert w.size == _lib.learned_weight_count(lmax)
    return w


def probes(w: workloads.Cluster, nrandom: int, seed: int, ctx) -> np.ndarray:
    """T b for plane waves along +z, +x, -y and oblique (both helicities mixed), plus random vectors."""
    k0 = w.k0
    s, c = np.sin(np.pi / 6), np.cos(np.pi / 6)
    kv = np.array([[0, 0, k0], [k0, 0, 0], [0, -k0, 0], [k0 * s, 0, k0 * c]], complex)
    pols = np.array([1, 0, 1, 0], np.int32)
    B = _lib.plane_wave_expansion(w.lmax, w.positions, kv, pols, ctx=ctx)
    T = _lib.mie_blocks(w.lmax, w.k0, w.radii, w.eps, ctx=ctx)
    M = 2 * w.lmax * (w.lmax + 2)
    deg = np.array([l for l in range(1, w.lmax + 1) for _ in range(2 * l + 1)])
    Bq = B.reshape(w.radii.size, M // 2, 2, B.shape[1])
    TB = np.einsum("nqab,nqbp->nqap", T[:, deg - 1], Bq).reshape(w.n, B.shape[1])
    rng = np.random.default_rng(seed)
    Rn = rng.standard_normal((w.n, nrandom)) + 1j * rng.standard_normal((w.n, nrandom))
    return np.asfortranarray(np.concatenate([TB, Rn], axis=1))


def validation_score(ctx, weights, clusters) -> tuple[int, float]:
    """Total GMRES(50) iterations to 1e-8 and summed relative residual of the learned
    preconditioner with these weights over the validation clusters."""
    ctx.set_learned_weights(weights, 3.0)
    its, res = 0, 0.0
    for c, b in clusters:
        cert = c.solve(b, rtol=1e-8, restart=50, max_iterations=400, preconditioner="learned").convergence[0]
        its += cert.iterations
        res += cert.residual_norm / cert.rhs_norm
    return its, res


def train(clusters: int = 8, steps: int = 300, lr: float = 3e-3, nrandom: int = 2, seed: int = 0, ctx=None,
          log=print, eval_every: int = 25, nvalid: int = 2):
    ctx = ctx or _lib.default_context()
    ctx.set_learned_weights(None, 0.0)
    problems, names = [], []
    for i in range(clusters):
        w = workloads.training_cluster(i)
        problems.append(_lib.LearnedProblem(w.lmax, w.k0, w.radii, w.eps, w.positions,
                                            probes(w, nrandom, 7000 + i, ctx), ctx=ctx))
        names.append(f"{w.radii.size} spheres")
    valid = []
    for v in range(nvalid):
        w = workloads.learned_cluster(seed=3000 + v, count=512)
        c = _lib.SphereCluster(w.lmax, w.k0, w.radii, w.eps, w.positions, ctx=ctx)
        valid.append((c, _lib.plane_wave_expansion(w.lmax, w.positions, w.kvecs, w.pols, ctx=ctx)[:, 0]))
    lmax = 3
    wts = init_weights(lmax, seed)
    nprobe = sum(p.nprobe for p in problems)
    score0 = validation_score(ctx, wts, valid)
    chosen = (score0, 0, wts.copy())
    log(f"step 0: validation iterations {score0[0]} (two-level)")

    def total(wv):
        loss, grad = 0.0, np.zeros_like(wv)
        for p in problems:
            l, g = p.loss_grad(wv)
            loss += l
            grad += g
        return loss / nprobe, grad / nprobe

    loss0, _ = total(wts)
    m, v = np.zeros_like(wts), np.zeros_like(wts)
    b1, b2, eps = 0.9, 0.999, 1e-8
    t0 = time.time()
    history = []
    for it in range(1, steps + 1):
        loss, g = total(wts)
        m = b1 * m + (1 - b1) * g
        v = b2 * v + (1 - b2) * g * g
        wts = wts - lr * (m / (1 - b1**it)) / (np.sqrt(v / (1 - b2**it)) + eps)
        if it % eval_every == 0 or it == steps:
            score = validation_score(ctx, wts, valid)
            history.append({"step": it, "loss": loss, "iterations": score[0], "residual": score[1]})
            if score < chosen[0]:
                chosen = (score, it, wts.copy())
            log(f"step {it}: mean probe loss {loss:.5g} (untrained {loss0:.5g}), validation iterations "
                f"{score[0]} (two-level {score0[0]}), {time.time() - t0:.1f} s")
    ctx.set_learned_weights(None, 0.0)
    for p in problems:
        p.close()
    improved = chosen[1] > 0 and chosen[0][0] < score0[0]
    return (chosen[2] if improved else None), {
        "loss_untrained": loss0, "clusters": names, "steps": steps, "probes": nprobe,
        "validation": {"clusters": [f"512 spheres, seed {3000 + i}" for i in range(nvalid)],
                       "two_level_iterations": score0[0], "chosen_step": chosen[1] if improved else 0,
                       "chosen_iterations": chosen[0][0] if improved else score0[0]},
        "history": history}


def write_inc(weights_by_lmax: dict, note: str, reach: float = 3.0) -> None:
    lines = [
        "// Trained weights of the graph network of the learned preconditioner per lmax (generated by",
        "// treams-rs_b200/treams_b200/train_precond.py; lmax without trained weights uses Theta = 1).",
        f"// {note}",
        f"constexpr double LEARNED_REACH = {float(reach)!r};  // near-field reach in sphere diameters",
        "inline std::vector<double> learned_weights(int lmax) {",
    ]
    for L, w in sorted(weights_by_lmax.items()):
        vals = ", ".join(repr(float(x)) for x in w)
        lines.append(f"    if (lmax == {L}) return {{{vals}}};")
    lines += ["    return {};", "}", ""]
    INC.write_text("\n".join(lines))


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--clusters", type=int, default=8)
    ap.add_argument("--steps", type=int, default=300)
    ap.add_argument("--lr", type=float, default=3e-3)
    ap.add_argument("--nrandom", type=int, default=2, help="random probe vectors per cluster")
    ap.add_argument("--eval-every", type=int, default=25, help="Adam steps between validation solves")
    ap.add_argument("--write", action="store_true", help="rewrite csrc/learned_weights.inc")
    ap.add_argument("--out", default=None, help="also write the weights and the training record to this JSON file")
    args = ap.parse_args()
    w, info = train(args.clusters, args.steps, args.lr, nrandom=args.nrandom, eval_every=args.eval_every)
    print(json.dumps(info))
    if args.out:
        pathlib.Path(args.out).write_text(json.dumps({"weights": None if w is None else list(map(float, w)), **info}))
    if args.write:
        val = info["validation"]
        if w is None:
            write_inc({}, f"{args.clusters} clusters, {args.steps} Adam steps: no step beat Theta = 1 on the "
                          f"validation clusters ({val['two_level_iterations']} GMRES iterations)")
        else:
            write_inc({3: w}, f"trained on {args.clusters} clusters, step {val['chosen_step']} of {args.steps}: "
                              f"{val['chosen_iterations']} validation GMRES iterations (two-level "
                              f"{val['two_level_iterations']})")


if __name__ == "__main__":
    main()
