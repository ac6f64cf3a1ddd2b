"""The LinearBench-shaped harness (alien_b200/linear_bench.py) on the GPU:
a system written to MatrixMarket files and read back solves exactly as the
same system given to the solver directly, and the default right-hand side is
b = 1 as in the reference's MatrixMarketProblem."""
import json

import numpy as np
import pytest

from alien_b200 import abi, linear_bench
from tests import problems

pytestmark = pytest.mark.gpu


def run_json(capsys, argv):
    rc = linear_bench.main(argv + ["--json"])
    return rc, json.loads(capsys.readouterr().out.strip().splitlines()[-1])


@pytest.mark.parametrize("solver,pc,extra", [("cg", "ilu0", []), ("bicgs", "filu0", ["--filu-solver-iter", "4"]),
                                             ("cg", "diag", ["--mixed"])])
def test_files_solve_like_the_direct_call(ctx, tmp_path, capsys, solver, pc, extra):
    P = problems.get("diffusion12")
    abi.write_matrix_market(P, tmp_path / "a.mtx", tmp_path / "b.mtx")
    rc, out = run_json(capsys, ["--matrix", str(tmp_path / "a.mtx"), "--rhs", str(tmp_path / "b.mtx"),
                                "--solver", solver, "--precond", pc] + extra)
    assert rc == 0 and out["converged"] and out["rows"] == P.n and out["nnz"] == P.nnz
    A = ctx.matrix(P.row_ptr, P.cols, P.vals, abi.FMT_CSR | abi.FMT_ELL | abi.FMT_F32)
    x = ctx.vector(P.n)
    if "--mixed" in extra:
        st = abi.Mixed(ctx, A, solver=solver, precond=pc, tol=1e-8).solve(ctx.vector(P.b), x)
        assert out["iterations"] == st.inner_iterations and out["outer_iterations"] == st.outer_iterations
    else:
        kw = dict(filu_solver_iter=4) if pc == "filu0" else {}
        st = abi.Solver(ctx, A, solver=solver, precond=pc, tol=1e-8, max_iter=1000, **kw).solve(ctx.vector(P.b), x)
        assert out["iterations"] == st.iterations
    assert out["true_rel_residual"] < 1e-7
    xs = x.download()
    assert out["solution"]["max"] == float(xs.max()) and out["solution"]["abs_min"] == float(np.abs(xs).min())


def test_default_rhs_is_ones_and_generator_source(tmp_path, capsys):
    P = problems.get("poisson16")
    abi.write_matrix_market(P, tmp_path / "p.mtx")
    rc, out = run_json(capsys, ["--matrix", str(tmp_path / "p.mtx"), "--precond", "ilu0"])
    assert rc == 0 and out["rhs"] == {"min": 1.0, "max": 1.0, "abs_min": 1.0, "abs_max": 1.0}
    rc, out = run_json(capsys, ["--problem", "poisson:16", "--precond", "diag", "--repeat", "2"])
    assert rc == 0 and out["rel_error_vs_x_true"] < 1e-6
