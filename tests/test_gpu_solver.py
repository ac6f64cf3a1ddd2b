"""Device-resident CG/BiCGStab vs the oracle (the reference templates' arithmetic).

Parity bar: same convergence flag, iteration count within +-2 (the dot
products differ only in summation tree), the first stop-test values within
1e-9 relative, and the solution:
  * CG: within 1e-10 relative of the oracle's;
  * BiCGStab: within 1e-5 relative.  BiCGStab amplifies the last-bit
    differences of its dot products: re-running the oracle's own BiCGStab with
    nothing changed but the dot summation order (numpy pairwise, or an exactly
    rounded fsum) moves the 16^3 Jacobi solution by 1.4e-7 and 2.9e-7 relative
    and the iteration count by one.  No device summation tree can meet a
    tighter bar against a sequential CPU sum; the reference's own result
    depends on its BLAS the same way.
Runs both the CUDA-graph loop and the host-driven loop.
"""
import json
from pathlib import Path

import numpy as np
import pytest

from alien_b200 import abi
from oracle import oracle as O
from tests import problems

pytestmark = pytest.mark.gpu

GOLDEN = json.loads((Path(__file__).parent / "golden" / "solves.json").read_text())


def gpu_solve(ctx, P, use_graph=True, variant=abi.SPMV_AUTO, x0=None, **kw):
    A = ctx.matrix(P.row_ptr, P.cols, P.vals)
    S = abi.Solver(ctx, A, spmv_variant=variant, use_graph=use_graph, **kw)
    b = ctx.vector(P.b)
    x = ctx.vector(np.zeros(P.n) if x0 is None else x0)
    st = S.solve(b, x)
    return st, x.download(), S.history()


X_TOL = {"cg": 1e-10, "bicgs": 1e-5}


def check_parity(st, x, hist, r, solver="cg"):
    assert st.succeeded == r.converged
    assert abs(st.iterations - r.iterations) <= 2, (st.iterations, r.iterations)
    if r.converged and (st.iterations == r.iterations or solver != "cg"):
        nx = max(np.linalg.norm(r.x), 1e-300)
        assert np.linalg.norm(x - r.x) / nx <= X_TOL[solver], np.linalg.norm(x - r.x) / nx
    m = min(hist.size, r.history.size, 10)
    np.testing.assert_allclose(hist[:m], r.history[:m], rtol=1e-9)


CASES = [
    ("poisson32", "cg", "diag"),  # the 32^3 Jacobi-PCG case: 105 iterations
    ("poisson16", "cg", "ilu0"),
    ("poisson16", "bicgs", "diag"),
    ("poisson16", "bicgs", "ilu0"),
    ("diffusion12", "cg", "diag"),
    ("diffusion12", "cg", "ilu0"),
    ("diffusion24", "cg", "ilu0"),
    ("diffusion24", "cg", "diag"),
    ("diffusion2d_31x9", "bicgs", "ilu0"),
    ("convdiff_10x11x12", "bicgs", "diag"),
    ("convdiff_10x11x12", "bicgs", "ilu0"),
    ("convdiff16", "bicgs", "ilu0"),
    ("ragged", "bicgs", "diag"),
    ("ragged", "cg", "none"),
]


@pytest.mark.parametrize("use_graph", [True, False])
@pytest.mark.parametrize("name,solver,pc", CASES)
def test_solver_parity(ctx, name, solver, pc, use_graph):
    P = problems.get(name)
    kw = dict(solver=solver, precond=pc, tol=1e-8, max_iter=1000)
    st, x, hist = gpu_solve(ctx, P, use_graph=use_graph, **kw)
    r = O.solve(P.row_ptr, P.cols, P.vals, P.b, **kw)
    check_parity(st, x, hist, r, solver)
    if r.converged:
        assert st.true_residual < 1e-7
    if name == "poisson32" and pc == "diag":
        assert st.iterations == 105


@pytest.mark.parametrize("name,factor", [("poisson16", 0.0), ("poisson16", 0.5), ("diffusion12", 0.0)])
def test_cg_chebyshev_parity(ctx, name, factor):
    P = problems.get(name)
    kw = dict(solver="cg", precond="cheb", tol=1e-6, max_iter=300, poly_factor=factor, poly_order=3,
              poly_factor_max_iter=20)
    st, x, hist = gpu_solve(ctx, P, **kw)
    r = O.solve(P.row_ptr, P.cols, P.vals, P.b, **kw)
    assert st.succeeded == r.converged
    assert abs(st.iterations - r.iterations) <= 2
    np.testing.assert_allclose(hist[:5], r.history[:5], rtol=1e-8)


@pytest.mark.parametrize("variant", [abi.SPMV_CSR_SCALAR, abi.SPMV_ELL])
def test_variants_agree_bitwise(ctx, variant):
    P = problems.get("diffusion24")
    st0, x0, _ = gpu_solve(ctx, P, variant=abi.SPMV_CSR_STAGED, solver="cg", precond="ilu0", tol=1e-8)
    st1, x1, _ = gpu_solve(ctx, P, variant=variant, solver="cg", precond="ilu0", tol=1e-8)
    assert st0.iterations == st1.iterations
    np.testing.assert_array_equal(x0, x1)


def test_repeated_solves_reuse_graph(ctx):
    P = problems.get("diffusion12")
    A = ctx.matrix(P.row_ptr, P.cols, P.vals)
    S = abi.Solver(ctx, A, solver="cg", precond="ilu0", tol=1e-8)
    b = ctx.vector(P.b)
    xs = []
    for _ in range(3):
        x = ctx.vector(P.n)
        st = S.solve(b, x)
        xs.append(x.download())
        assert st.succeeded
    np.testing.assert_array_equal(xs[0], xs[1])
    np.testing.assert_array_equal(xs[0], xs[2])


def test_null_rhs_and_iteration_limits(ctx):
    P = problems.get("poisson16")
    A = ctx.matrix(P.row_ptr, P.cols, P.vals)
    S = abi.Solver(ctx, A, solver="cg", precond="diag", tol=1e-8)
    st = S.solve(ctx.vector(P.n), ctx.vector(P.n))
    assert st.succeeded and st.iterations == 0  # Iteration::nullRhs
    for case in [c for c in GOLDEN["cases"] if c["max_iter"] <= 1]:
        Q = problems.get(case["problem"])
        st, x, hist = gpu_solve(ctx, Q, solver=case["solver"], precond=case["precond"], tol=case["tol"],
                                max_iter=case["max_iter"])
        assert st.iterations == case["iterations"] and st.succeeded == case["converged"]


@pytest.mark.parametrize("case", [c for c in GOLDEN["cases"] if c["precond"] != "cheb" and c["converged"]],
                         ids=lambda c: f"{c['problem']}-{c['solver']}-{c['precond']}")
def test_golden_iteration_counts(ctx, case):
    """Converged golden cases recorded from Alien's own templates."""
    P = problems.get(case["problem"])
    st, x, hist = gpu_solve(ctx, P, solver=case["solver"], precond=case["precond"], tol=case["tol"],
                            max_iter=case["max_iter"])
    assert st.succeeded
    assert abs(st.iterations - case["iterations"]) <= 2
    xs = np.array([float.fromhex(v) for v in case["x_sample"]])
    np.testing.assert_allclose(x[case["x_index"]], xs, rtol=0, atol=X_TOL[case["solver"]] * np.max(np.abs(xs)))


def test_initial_guess_is_used(ctx):
    P = problems.get("diffusion12")
    x0 = np.random.default_rng(0).uniform(-1, 1, P.n)
    kw = dict(solver="bicgs", precond="ilu0", tol=1e-9, max_iter=200)
    st, x, hist = gpu_solve(ctx, P, x0=x0, **kw)
    r = O.solve(P.row_ptr, P.cols, P.vals, P.b, x0=x0, **kw)
    check_parity(st, x, hist, r, "bicgs")


def test_breakdown_reported(ctx):
    """The zero operator: p.Ap == 0 on the first step, the stop test fails, so
    CG throws NullValueException("alpha") (CG.h:96-104); BiCGStab's v.r0 == 0
    throws "alpha" too (BiCGStab.h:186-187)."""
    n = 64
    rp = np.arange(n + 1, dtype=np.int32)
    ci = np.arange(n, dtype=np.int32)
    vals = np.zeros(n)
    P = abi.CsrProblem(n, rp, ci, vals, np.ones(n), np.ones(n), None, (n, 1, 1))
    for solver in ("cg", "bicgs"):
        st, x, hist = gpu_solve(ctx, P, solver=solver, precond="none", tol=1e-8, max_iter=10)
        r = O.solve(rp, ci, vals, np.ones(n), solver=solver, precond="none", tol=1e-8, max_iter=10)
        assert r.error == -3 and r.breakdown == "alpha"
        assert st.error == abi.AB2_ERR_BREAKDOWN and st.breakdown == "alpha"
        assert st.iterations == r.iterations and not st.succeeded
