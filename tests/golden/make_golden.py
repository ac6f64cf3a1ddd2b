"""Regenerates tests/golden/*.json from Alien's OWN Krylov templates.

    python tests/golden/make_golden.py

Runs oracle/_ref/libalien_ref.so (the reference's header-only CG.h,
BiCGStab.h, Iteration.h, DiagPreconditioner.h, ILU0Preconditioner.h,
ChebyshevPreconditioner.h, FILU0Preconditioner.h and
NeumannPolyPreconditioner.h compiled over a SimpleCSR-restating CPU algebra,
see oracle/ref/ref_driver.cpp) on small seeded systems from libab2's generators and
records, per case: iteration count, convergence flag, breakdown, the full
residual history of the stop test, and the solution (as float64 hex, so the
fixture is exact).  The inputs are regenerated from their seeds by the tests.
"""
from __future__ import annotations

import hashlib
import json
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from alien_b200 import abi  # noqa: E402  (generators only: host code)
from oracle import oracle as O  # noqa: E402

OUT = Path(__file__).resolve().parent / "solves.json"

PROBLEMS = {
    "poisson16": lambda: abi.poisson(16, 16, 16, seed=0),
    "poisson2d_23x17": lambda: abi.poisson(23, 17, 1, seed=3),
    "diffusion12": lambda: abi.diffusion(12, 12, 12, sigma=1.0, smooth=2.0, seed=1),
    "diffusion2d_31x9": lambda: abi.diffusion(31, 9, 1, sigma=1.5, smooth=3.0, seed=7),
    "convdiff_10x11x12": lambda: abi.convdiff(10, 11, 12, peclet=10.0, modes=8, seed=2),
}

CASES = []
for prob in PROBLEMS:
    for solver in ("cg", "bicgs"):
        for pc in ("diag", "ilu0", "cheb"):
            CASES.append(dict(problem=prob, solver=solver, precond=pc, tol=1e-8, max_iter=300, poly_factor=0.0,
                              poly_order=3, poly_factor_max_iter=20, cheb_saad=False))
        # ChebyshevPreconditioner<AlgebraT, true> (Saad's recurrence, _algo1)
        CASES.append(dict(problem=prob, solver=solver, precond="cheb", tol=1e-8, max_iter=300, poly_factor=0.0,
                          poly_order=3, poly_factor_max_iter=20, cheb_saad=True))
# FILU0 (nonsymmetric sweeps: BiCGStab) and Neumann (omega = 1 / the
# Gershgorin bound of each matrix, passed explicitly: the reference's own
# estimate draws from std::random_device)
GERSHGORIN = {}
for prob in PROBLEMS:
    for fi, si in ((0, 3), (1, 2), (0, 1)):
        CASES.append(dict(problem=prob, solver="bicgs", precond="filu0", tol=1e-8, max_iter=300, poly_factor=0.0,
                          poly_order=3, poly_factor_max_iter=10, filu_factor_iter=fi, filu_solver_iter=si))
    CASES.append(dict(problem=prob, solver="cg", precond="neumann", tol=1e-8, max_iter=300, poly_factor="1/gershgorin",
                      poly_order=3, poly_factor_max_iter=10))
# edge cases the reference's control flow has
CASES += [
    dict(problem="poisson16", solver="cg", precond="diag", tol=1e-8, max_iter=1, poly_factor=0.0, poly_order=3,
         poly_factor_max_iter=10),
    dict(problem="poisson16", solver="bicgs", precond="diag", tol=1e-8, max_iter=0, poly_factor=0.0, poly_order=3,
         poly_factor_max_iter=10),
    dict(problem="poisson16", solver="cg", precond="cheb", tol=1e-6, max_iter=200, poly_factor=0.5, poly_order=3,
         poly_factor_max_iter=10),
    dict(problem="poisson16", solver="bicgs", precond="ilu0", tol=1e-3, max_iter=100, poly_factor=0.0, poly_order=3,
         poly_factor_max_iter=10),
]


def hexs(a: np.ndarray) -> list[str]:
    return [float(v).hex() for v in a]


def main() -> int:
    if not O.ref_available():
        print("oracle/_ref/libalien_ref.so is missing: run make -f oracle/Makefile with the reference sources")
        return 1
    cache = {k: f() for k, f in PROBLEMS.items()}
    out = {"generator": "libab2 ab2_problem_* (include/ab2_problems.h)", "problems": {}, "cases": []}
    for k, P in cache.items():
        out["problems"][k] = dict(n=P.n, nnz=P.nnz, shape=list(P.shape),
                                  vals_sha256=hashlib.sha256(P.vals.tobytes()).hexdigest(),
                                  b_sha256=hashlib.sha256(P.b.tobytes()).hexdigest())
    for c in CASES:
        P = cache[c["problem"]]
        if c["poly_factor"] == "1/gershgorin":
            c["poly_factor"] = 1.0 / float(np.add.reduceat(np.abs(P.vals), P.row_ptr[:-1]).max())
        kw = {k: v for k, v in c.items() if k != "problem"}
        r = O.solve(P.row_ptr, P.cols, P.vals, P.b, which="ref", **kw)
        idx = np.unique(np.linspace(0, P.n - 1, 48).astype(np.int64))
        out["cases"].append(dict(**c, iterations=r.iterations, converged=r.converged, breakdown=r.breakdown,
                                 history_len=int(r.history.size),
                                 history_sha256=hashlib.sha256(r.history.tobytes()).hexdigest(),
                                 history_head=hexs(r.history[:12]), history_tail=hexs(r.history[-4:]),
                                 x_sha256=hashlib.sha256(r.x.tobytes()).hexdigest(),
                                 x_index=idx.tolist(), x_sample=hexs(r.x[idx]),
                                 x_norm2=float(np.linalg.norm(r.x)).hex()))
        print(c["problem"], c["solver"], c["precond"], r.iterations, r.converged)
    OUT.write_text(json.dumps(out, indent=0))
    print("wrote", OUT, OUT.stat().st_size, "bytes")
    return 0


if __name__ == "__main__":
    sys.exit(main())
