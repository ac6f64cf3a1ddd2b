"""The CPU oracle, pinned (no GPU needed).

* the known-answer checks of Alien's own algebra test
  (src/refsemantic/tests/TestMVExpr.cc:105-167) hold for the oracle algebra;
* the restatement (oracle/ab2_oracle.cpp) reproduces, bit for bit, the solves
  recorded in tests/golden/solves.json from Alien's own Krylov templates
  (oracle/_ref, generated by tests/golden/make_golden.py);
* when oracle/_ref is present, restatement and reference templates agree on
  further random systems too.
"""
import hashlib
import json
from pathlib import Path

import numpy as np
import pytest

from oracle import oracle as O
from tests import problems

GOLDEN = json.loads((Path(__file__).parent / "golden" / "solves.json").read_text())


def unhex(a):
    return np.array([float.fromhex(v) for v in a])


# ----------------------------------------------------------------- TestMVExpr KATs
def test_testmvexpr_known_answers():
    rp, ci, v = problems.laplacian_1d(10)
    n, lam = 10, 0.5
    x = np.ones(n)
    nrm = lambda a: np.sqrt(O.dot(a, a))  # norm2 = sqrt(dot), CBLASMPIKernel.h:113-124
    assert nrm(x) == np.sqrt(10)
    y = lam * x
    assert nrm(y) == np.sqrt(10 * 0.25)
    y = O.spmv(rp, ci, v, x)
    assert nrm(y) == np.sqrt(2)
    r = y - O.spmv(rp, ci, v, x)
    assert nrm(r) == 0.0
    y = y + lam * x
    assert nrm(y) == np.sqrt(2 * 1.5 * 1.5 + (n - 2) * 0.25)
    y = O.spmv(rp, ci, v, lam * x)
    assert nrm(y) == np.sqrt(0.5)
    y = np.arange(n, dtype=np.float64)
    assert O.dot(x, y) == 45
    assert O.dot(lam * x, y) == 22.5
    assert O.dot(x, r + y) == 45
    assert O.dot(x, O.spmv(rp, ci, v, y)) == 9
    # ||lambda A||_F = lambda ||A||_F
    assert np.sqrt(O.dot(lam * v, lam * v)) == lam * np.sqrt(O.dot(v, v))


# ----------------------------------------------------------------- golden solves
@pytest.mark.parametrize("case", GOLDEN["cases"], ids=lambda c: f"{c['problem']}-{c['solver']}-{c['precond']}-m{c['max_iter']}")
def test_restatement_matches_reference_templates(case):
    P = problems.get(case["problem"])
    meta = GOLDEN["problems"][case["problem"]]
    assert hashlib.sha256(P.vals.tobytes()).hexdigest() == meta["vals_sha256"]
    assert hashlib.sha256(P.b.tobytes()).hexdigest() == meta["b_sha256"]
    kw = {k: case[k] for k in ("solver", "precond", "tol", "max_iter", "poly_factor", "poly_order",
                               "poly_factor_max_iter")}
    kw["cheb_saad"] = case.get("cheb_saad", False)
    kw["filu_factor_iter"] = case.get("filu_factor_iter", 0)
    kw["filu_solver_iter"] = case.get("filu_solver_iter", 3)
    r = O.solve(P.row_ptr, P.cols, P.vals, P.b, which="oracle", **kw)
    assert r.iterations == case["iterations"]
    assert r.converged == case["converged"]
    assert r.breakdown == case["breakdown"]
    assert r.history.size == case["history_len"]
    assert hashlib.sha256(r.history.tobytes()).hexdigest() == case["history_sha256"]
    assert hashlib.sha256(r.x.tobytes()).hexdigest() == case["x_sha256"]
    np.testing.assert_array_equal(r.x[case["x_index"]], unhex(case["x_sample"]))


@pytest.mark.skipif(not O.ref_available(), reason="oracle/_ref not built")
@pytest.mark.parametrize("seed", [0, 1, 2])
@pytest.mark.parametrize("solver,pc", [("cg", "diag"), ("bicgs", "ilu0"), ("bicgs", "diag"), ("cg", "ilu0"),
                                       ("bicgs", "cheb")])
def test_restatement_vs_reference_random(seed, solver, pc):
    P = problems.ragged(300 + 37 * seed, seed=100 + seed)
    kw = dict(solver=solver, precond=pc, tol=1e-10, max_iter=60, poly_factor=0.0, poly_order=3,
              poly_factor_max_iter=8)
    a = O.solve(P.row_ptr, P.cols, P.vals, P.b, which="oracle", **kw)
    r = O.solve(P.row_ptr, P.cols, P.vals, P.b, which="ref", **kw)
    assert a.iterations == r.iterations and a.converged == r.converged
    np.testing.assert_array_equal(a.x, r.x)
    np.testing.assert_array_equal(a.history, r.history)


@pytest.mark.skipif(not O.ref_available(), reason="oracle/_ref not built")
@pytest.mark.parametrize("name", ["poisson16", "diffusion12", "convdiff_10x11x12", "ragged"])
def test_ilu0_and_chebyshev_vs_reference(name):
    P = problems.get(name)
    np.testing.assert_array_equal(O.ilu0_factor(P.row_ptr, P.cols, P.vals, "oracle"),
                                  O.ilu0_factor(P.row_ptr, P.cols, P.vals, "ref"))
    np.testing.assert_array_equal(O.ilu0_apply(P.row_ptr, P.cols, P.vals, P.b, "oracle"),
                                  O.ilu0_apply(P.row_ptr, P.cols, P.vals, P.b, "ref"))
    for saad in (False, True):
        np.testing.assert_array_equal(O.cheb_apply(P.row_ptr, P.cols, P.vals, P.b, 0.0, 3, 12, "oracle", saad=saad),
                                      O.cheb_apply(P.row_ptr, P.cols, P.vals, P.b, 0.0, 3, 12, "ref", saad=saad))


def test_lanczos_bounds_bracket_the_spectrum():
    """Lanczos bounds (no reference counterpart): the Ritz interval lies inside
    the spectrum of D^-1 A, the upper bound is widened by 10%."""
    P = problems.get("diffusion12")
    A = np.zeros((P.n, P.n))
    for r in range(P.n):
        A[r, P.cols[P.row_ptr[r]:P.row_ptr[r + 1]]] = P.vals[P.row_ptr[r]:P.row_ptr[r + 1]]
    s = 1.0 / np.sqrt(np.diag(A))
    ev = np.linalg.eigvalsh(s[:, None] * A * s[None, :])
    a, b = O.cheb_bounds(P.row_ptr, P.cols, P.vals, 0.0, 20, lanczos=True)
    assert ev[0] <= a <= ev[-1]
    assert ev[-1] <= b <= 1.1 * ev[-1] * (1 + 1e-12)
    assert abs(b / 1.1 - ev[-1]) < 1e-3 * ev[-1]


def test_krylov_config1_iteration_count():
    """32^3 Poisson, b = A x_true (seed 0), Jacobi-PCG to 1e-8."""
    P = problems.get("poisson32")
    r = O.solve(P.row_ptr, P.cols, P.vals, P.b, solver="cg", precond="diag", tol=1e-8, max_iter=1000)
    assert r.converged and r.iterations == 105
    assert np.linalg.norm(r.x - P.x_true) / np.linalg.norm(P.x_true) < 1e-6


def test_ell_layout_matches_csr():
    P = problems.get("ragged")
    off, ec, ev = O.ell_layout(P.row_ptr, P.cols, P.vals, 32)
    n = P.n
    for row in range(0, n, 37):
        s, lane = divmod(row, 32)
        w = off[s + 1] - off[s]
        slots = off[s] * 32 + np.arange(w) * 32 + lane
        a, b = P.row_ptr[row], P.row_ptr[row + 1]
        assert np.array_equal(ec[slots][: b - a], P.cols[a:b])
        assert np.array_equal(ev[slots][: b - a], P.vals[a:b])
        assert np.all(ev[slots][b - a:] == 0)


# ----------------------------------------------------------------- mixed precision (no reference counterpart)
@pytest.mark.parametrize("name,solver,pc", [("poisson16", "cg", "diag"), ("poisson16", "cg", "ilu0"),
                                            ("convdiff_10x11x12", "bicgs", "ilu0"), ("ragged", "bicgs", "diag")])
def test_mixed_refinement_restatement(name, solver, pc):
    """The FP32-inner / FP64-refinement restatement reaches the FP64 tolerance,
    each step cuts the true residual by about the inner tolerance, and the
    result agrees with a plain FP64 solve."""
    P = problems.get(name)
    r = O.mixed_solve(P.row_ptr, P.cols, P.vals, P.b, solver=solver, precond=pc, tol=1e-10, inner_tol=1e-4)
    assert r.succeeded and r.error == 0 and r.true_residual < 1e-10
    assert r.history[0] == 1.0 and np.all(np.diff(r.history) < 0)
    assert r.outer_iterations <= 4
    x64 = O.solve(P.row_ptr, P.cols, P.vals, P.b, solver=solver, precond="ilu0", tol=1e-13, max_iter=5000).x
    assert np.linalg.norm(r.x - x64) / np.linalg.norm(x64) < 1e-8


def test_fp32_pieces_are_float_restatements():
    """FP32 SpMV and tree dot equal the same sums done in numpy float32 with
    the same order (row-sequential SpMV; the tree for the dot)."""
    P = problems.get("diffusion12")
    x = np.random.default_rng(1).uniform(-1, 1, P.n).astype(np.float32)
    y = O.spmv32(P.row_ptr, P.cols, P.vals, x)
    v32 = P.vals.astype(np.float32)
    for i in range(0, P.n, 97):
        acc = np.float32(0)
        for k in range(P.row_ptr[i], P.row_ptr[i + 1]):
            acc = np.float32(acc + np.float32(v32[k] * x[P.cols[k]]))
        assert acc == y[i]
    d = O.dot_tree32(x, x, 1184)
    assert abs(float(d) - float(np.dot(x.astype(np.float64), x.astype(np.float64)))) < 1e-5 * float(d)
    # FP32 ILU(0) application is close to the FP64 one
    z32 = O.ilu0_apply32(P.row_ptr, P.cols, P.vals, x)
    z64 = O.ilu0_apply(P.row_ptr, P.cols, P.vals, x.astype(np.float64))
    assert np.max(np.abs(z32 - z64)) < 1e-5 * np.max(np.abs(z64))


# ----------------------------------------------------------------- FILU0 and Neumann
@pytest.mark.skipif(not O.ref_available(), reason="oracle/_ref not built")
@pytest.mark.parametrize("name", ["poisson16", "diffusion12", "convdiff16", "ragged", "diffusion2d_31x9"])
def test_filu0_and_neumann_vs_reference(name):
    """FILU0Preconditioner.h (factor by 0, 1 or 3 fixed-point sweeps -- each
    starting from the previous iterate, as the reference's init hands its own
    factor matrix to factorizeMultiIter -- and 0, 1 or 3 Jacobi sweeps per
    triangle, device-algebra branch) and NeumannPolyPreconditioner.h: factor
    and application bit for bit."""
    P = problems.get(name)
    y = np.random.default_rng(5).normal(size=P.n)
    for fi in (0, 1, 3):
        for si in (0, 1, 3):
            xo, luo = O.filu0_apply(P.row_ptr, P.cols, P.vals, y, fi, si, "oracle")
            xr, lur = O.filu0_apply(P.row_ptr, P.cols, P.vals, y, fi, si, "ref")
            np.testing.assert_array_equal(luo, lur)
            np.testing.assert_array_equal(xo, xr)
    if name != "ragged":
        _, lu_ilu = O.filu0_apply(P.row_ptr, P.cols, P.vals, y, 0, 1, "oracle")
        np.testing.assert_array_equal(lu_ilu, O.ilu0_factor(P.row_ptr, P.cols, P.vals))
    omega = 1.0 / float(np.add.reduceat(np.abs(P.vals), P.row_ptr[:-1]).max())
    for order in (0, 1, 3):
        yo, wo = O.neumann_apply(P.row_ptr, P.cols, P.vals, y, omega, order, 10, "oracle")
        yr, _ = O.neumann_apply(P.row_ptr, P.cols, P.vals, y, omega, order, 10, "ref")
        assert wo == omega
        np.testing.assert_array_equal(yo, yr)


def test_neumann_power_method_estimates_the_largest_eigenvalue():
    """computeFactor's unnormalised power iteration approaches lambda_max
    from below (slowly: lambda_2/lambda_1 is close to 1)."""
    P = problems.get("poisson16")
    lam = 6 + 6 * np.cos(np.pi / 17)  # 3-D 7-point Dirichlet Laplacian, 16^3 cells
    est = [1 / O.neumann_apply(P.row_ptr, P.cols, P.vals, np.ones(P.n), 0.0, 3, it)[1] for it in (10, 40)]
    assert est[0] < est[1] < lam and (lam - est[1]) / lam < 0.05
