"""Solve a linear system from MatrixMarket files (or a seeded generator) on
the GPU and report what Alien's LinearBench reports.

The reference's harness (benchmark/src/alien/benchmark/LinearBench.cpp and
MatrixMarketProblem.cpp) reads a matrix and an optional right-hand side
(b = 1 without one), solves from x = 0 with the chosen solver, and prints the
solution's and the right-hand side's analytics (min, max, min |.|, max |.|:
VectorAnalytics.cpp) and the residual.  Same here, through libab2's public
API: the matrix is read on the host (ab2_problem_read_matrix_market), copied
to the device, the solver is set up and run device-resident, and the
timings come from the library's CUDA events.

    python -m alien_b200.linear_bench --matrix A.mtx [--rhs b.mtx] --solver cg --precond ilu0
    python -m alien_b200.linear_bench --problem diffusion:64 --precond filu0 --solver bicgs --json
"""
from __future__ import annotations

import argparse
import json
import sys
import time

import numpy as np

from alien_b200 import abi


def analytics(v: np.ndarray) -> dict:
    a = np.abs(v)
    return {"min": float(v.min()), "max": float(v.max()), "abs_min": float(a.min()), "abs_max": float(a.max())}


def load(args) -> tuple[abi.CsrProblem, str]:
    if args.matrix:
        return abi.read_matrix_market(args.matrix, args.rhs), args.matrix
    kind, _, size = args.problem.partition(":")
    m = int(size or 32)
    gen = {"poisson": lambda: abi.poisson(m, m, m, seed=args.seed),
           "diffusion": lambda: abi.diffusion(m, m, m, sigma=1.0, smooth=4.0, seed=args.seed),
           "convdiff": lambda: abi.convdiff(m, m, m, peclet=10.0, modes=8, seed=args.seed)}
    if kind not in gen:
        raise SystemExit(f"unknown problem {kind!r} (poisson, diffusion, convdiff)")
    return gen[kind](), f"{kind}:{m} seed {args.seed}"


def run(args) -> dict:
    t0 = time.perf_counter()
    P, source = load(args)
    t_load = time.perf_counter() - t0
    ctx = abi.Context(args.device)
    t0 = time.perf_counter()
    fmts = abi.FMT_CSR | abi.FMT_ELL | (abi.FMT_F32 if args.mixed else 0)
    A = ctx.matrix(P.row_ptr, P.cols, P.vals, fmts)
    b = ctx.vector(P.b)
    ctx.synchronize()
    t_upload = time.perf_counter() - t0
    opts = dict(solver=args.solver, precond=args.precond, tol=args.tol, poly_factor=args.poly_factor,
                poly_order=args.poly_order, poly_factor_max_iter=args.poly_max_iter,
                filu_factor_iter=args.filu_factor_iter, filu_solver_iter=args.filu_solver_iter)
    runs = []
    for _ in range(max(1, args.repeat)):
        x = ctx.vector(P.n)
        if args.mixed:
            S = abi.Mixed(ctx, A, max_outer=args.max_outer, inner_tol=args.inner_tol, inner_max_iter=args.max_iter,
                          **opts)
            st = S.solve(b, x)
            rec = {"converged": bool(st.succeeded), "outer_iterations": st.outer_iterations,
                   "iterations": st.inner_iterations, "setup_ms": st.setup_ms, "solve_ms": st.solve_ms,
                   "true_rel_residual": st.true_residual}
        else:
            S = abi.Solver(ctx, A, max_iter=args.max_iter, **opts)
            st = S.solve(b, x)
            rec = {"converged": bool(st.succeeded), "iterations": st.iterations, "setup_ms": st.setup_ms,
                   "solve_ms": st.solve_ms, "residual": st.residual, "true_rel_residual": st.true_residual,
                   "breakdown": st.breakdown}
        S.close()
        runs.append((rec, x))
    rec, x = min(runs, key=lambda r: r[0]["setup_ms"] + r[0]["solve_ms"])
    xs = x.download()
    r = ctx.vector(P.n)
    ctx.mult(A, x, r)
    res = P.b - r.download()
    out = {"source": source, "rows": P.n, "nnz": P.nnz, "solver": args.solver, "precond": args.precond,
           "precision": "fp32 inner / fp64 refinement" if args.mixed else "fp64", "tol": args.tol,
           "load_s": round(t_load, 4), "upload_s": round(t_upload, 4), **rec,
           "residual_norm2": float(np.linalg.norm(res)), "solution": analytics(xs), "rhs": analytics(P.b)}
    if P.x_true is not None:
        out["rel_error_vs_x_true"] = float(np.linalg.norm(xs - P.x_true) / np.linalg.norm(P.x_true))
    if args.write_solution:
        np.savetxt(args.write_solution, xs)
    return out


def parser() -> argparse.ArgumentParser:
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    src = ap.add_mutually_exclusive_group(required=True)
    src.add_argument("--matrix", help="MatrixMarket coordinate real file")
    src.add_argument("--problem", help="seeded generator instead: poisson:N, diffusion:N or convdiff:N")
    ap.add_argument("--rhs", help="MatrixMarket array real right-hand side (default b = 1)")
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--solver", default="cg", choices=["cg", "bicgs"])
    ap.add_argument("--precond", default="diag", choices=sorted(abi.PRECOND))
    ap.add_argument("--tol", type=float, default=1e-8)
    ap.add_argument("--max-iter", type=int, default=1000)
    ap.add_argument("--poly-factor", type=float, default=0.0)
    ap.add_argument("--poly-order", type=int, default=3)
    ap.add_argument("--poly-max-iter", type=int, default=20)
    ap.add_argument("--filu-factor-iter", type=int, default=0)
    ap.add_argument("--filu-solver-iter", type=int, default=3)
    ap.add_argument("--mixed", action="store_true", help="FP32 inner solver inside FP64 refinement")
    ap.add_argument("--max-outer", type=int, default=20)
    ap.add_argument("--inner-tol", type=float, default=1e-4)
    ap.add_argument("--repeat", type=int, default=1, help="solves; the fastest is reported")
    ap.add_argument("--device", type=int, default=0)
    ap.add_argument("--write-solution", help="text file for x")
    ap.add_argument("--json", action="store_true", help="one JSON line instead of the text report")
    return ap


def main(argv=None) -> int:
    args = parser().parse_args(argv)
    out = run(args)
    if args.json:
        print(json.dumps(out))
    else:
        for k, v in out.items():
            print(f"{k:22s} {v}")
    return 0 if out["converged"] else 1


if __name__ == "__main__":
    sys.exit(main())
