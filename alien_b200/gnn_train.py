"""Training of the learned preconditioner on the GPU (libab2's own kernels).

Training data are (residual, error) pairs that the plain FP64 CG + ILU(0)
solver itself produces: for each seeded coefficient field (heterogeneous 3-D
7-point diffusion, log10 k ~ smoothed N(0, sigma^2), smoothing length drawn in
[2, 8] cells) the solver runs to 1e-12 for the reference solution x*, and
again for k = 0, 2, 5, 10, 20, ... iterations from x = 0; each iterate x_k
gives r_k = b - A x_k and e_k = x* - x_k.  Every step is one Adam update on
one pair through ab2_gnn_train_step (forward, loss (z-e)^T A (z-e)/e^T A e,
backward and the optimiser all run on the device).

    python -m alien_b200.gnn_train --fields 64 --side 64 --out alien_b200/gnn_weights.npy
"""
from __future__ import annotations

import argparse
import json
import time
from pathlib import Path

import numpy as np

from alien_b200 import abi

ITERATES = (0, 2, 5, 10, 20, 40)


def field(side: int, seed: int, sigma: float = 1.5, lengths=(2.0, 8.0)) -> abi.CsrProblem:
    """One training or test field; the smoothing length is drawn from the seed."""
    u = 0.5 * (abi.lib().ab2_rng_uniform(seed, 77, 0) + 1.0)
    return abi.diffusion(side, side, side, sigma=sigma, smooth=lengths[0] + u * (lengths[1] - lengths[0]), seed=seed)


def pairs(ctx: abi.Context, P: abi.CsrProblem, A: abi.Matrix, iterates=ITERATES):
    """(r_k, e_k) host arrays from CG + ILU(0) iterates of one system."""
    b = ctx.vector(P.b)
    x = ctx.vector(P.n)
    S = abi.Solver(ctx, A, solver="cg", precond="ilu0", tol=1e-12, max_iter=5000)
    S.solve(b, x)
    xstar = x.download()
    S.close()
    ax = ctx.vector(P.n)
    out = []
    for k in iterates:
        xk = np.zeros(P.n)
        if k > 0:
            Sk = abi.Solver(ctx, A, solver="cg", precond="ilu0", tol=0.0, max_iter=k)
            ctx.assign(x, 0.0)
            Sk.solve(b, x)
            Sk.close()
            xk = x.download()
        x.upload(xk)
        ctx.mult(A, x, ax)
        r = P.b - ax.download()
        e = xstar - xk
        if np.linalg.norm(e) > 0:
            out.append((r, e))
    for v in (b, x, ax):
        v.close()
    return out


def train(ctx: abi.Context, net: abi.Gnn, fields: int = 64, side: int = 64, steps_per_pair: int = 4,
          lr: float = 1e-3, seed: int = 1000, iterates=ITERATES, log_every: int = 0,
          lr_final: float | None = None) -> list[float]:
    """Trains `net` in place; returns the loss of every step.  The learning
    rate decays geometrically from lr to lr_final over the fields."""
    hist: list[float] = []
    t0 = time.perf_counter()
    lr0 = lr
    for f in range(fields):
        if lr_final is not None and fields > 1:
            lr = lr0 * (lr_final / lr0) ** (f / (fields - 1))
        P = field(side, seed + f)
        A = ctx.matrix(P.row_ptr, P.cols, P.vals)
        net.bind(A)
        data = pairs(ctx, P, A, iterates)
        vr, ve = ctx.vector(P.n), ctx.vector(P.n)
        order = np.random.default_rng(seed + f).permutation(len(data) * steps_per_pair) % len(data)
        for k in order:
            r, e = data[k]
            vr.upload(r)
            ve.upload(e)
            hist.append(net.train_step(vr, ve, lr))
        if log_every and (f + 1) % log_every == 0:
            print(f"field {f + 1}/{fields}: mean loss of its steps {np.mean(hist[-len(order):]):.4f} "
                  f"({time.perf_counter() - t0:.1f} s)", flush=True)
        vr.close()
        ve.close()
    return hist


def main() -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--fields", type=int, default=64)
    ap.add_argument("--side", type=int, default=64)
    ap.add_argument("--steps-per-pair", type=int, default=4)
    ap.add_argument("--lr", type=float, default=1e-3)
    ap.add_argument("--lr-final", type=float, default=1e-4)
    ap.add_argument("--seed", type=int, default=1000)
    ap.add_argument("--init-seed", type=int, default=0)
    ap.add_argument("--out", default=str(Path(__file__).resolve().parent / "gnn_weights.npy"))
    a = ap.parse_args()
    ctx = abi.Context(0)
    net = abi.Gnn(ctx, None, seed=a.init_seed)  # libab2's seeded He-style initialisation
    t = time.perf_counter()
    hist = train(ctx, net, a.fields, a.side, a.steps_per_pair, a.lr, a.seed, log_every=max(1, a.fields // 16),
                 lr_final=a.lr_final)
    elapsed = time.perf_counter() - t
    np.save(a.out, net.params)
    n = max(1, len(hist) // 20)
    chunks = np.array_split(np.asarray(hist), 20)
    summary = {"fields": a.fields, "side": a.side, "field_seeds": [a.seed, a.seed + a.fields - 1],
               "sigma": 1.5, "smoothing_length": [2.0, 8.0], "iterates": list(ITERATES),
               "steps_per_pair": a.steps_per_pair, "steps": len(hist), "lr": [a.lr, a.lr_final], "optimizer": "adam",
               "init_seed": a.init_seed, "seconds": round(elapsed, 1),
               "loss_mean_by_twentieth": [round(float(c.mean()), 4) for c in chunks if c.size]}
    Path(a.out).with_suffix(".json").write_text(json.dumps(summary, indent=1) + "\n")
    print(f"trained {len(hist)} steps on {a.fields} fields of {a.side}^3 in {elapsed:.1f} s; "
          f"loss first {np.mean(hist[:n]):.4f} last {np.mean(hist[-n:]):.4f}; weights -> {a.out}")
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
