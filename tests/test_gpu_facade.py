"""libab2 behind Alien's own back-end interfaces (IInternalLinearAlgebra,
IInternalLinearSolver, AlgebraTraits<BackEnd::tag::b200>).

tests/cpp/facade is include/alien/b200/backend.h compiled against the
reference's core/backend/{BackEnd,IInternalLinearAlgebraT,
IInternalLinearSolverT}.h and expression/solver/{ILinearSolver,SolverStat}.h
(SolverStat.cc linked from the reference); it calls every operation through
the virtual interfaces, as Alien's LinearAlgebra<Tag> / LinearSolver<Tag>
facades do, after converting the system the way the simplecsr -> b200
converters do.  The results must equal the oracle's: the algebra bit for bit
(dot and norms: the reduction tree), the solver bit for bit against the
oracle summing its dots in libab2's tree.  Skipped when the binary was not
built (no reference sources).
"""
import json
import subprocess
from pathlib import Path

import numpy as np
import pytest

from oracle import oracle as O
from tests import problems

pytestmark = pytest.mark.gpu

BIN = Path(__file__).resolve().parent / "cpp" / "_build" / "facade"
needs_bin = pytest.mark.skipif(not BIN.exists(), reason="tests/cpp/_build/facade not built (reference sources absent)")


def write_system(P, d: Path):
    P.row_ptr.astype(np.int32).tofile(d / "rp.i32")
    P.cols.astype(np.int32).tofile(d / "ci.i32")
    P.vals.astype(np.float64).tofile(d / "v.f64")
    P.b.astype(np.float64).tofile(d / "b.f64")


def f64(d: Path, name: str) -> np.ndarray:
    return np.fromfile(d / name, dtype=np.float64)


@needs_bin
@pytest.mark.parametrize("name", ["diffusion12", "convdiff_10x11x12", "ragged"])
def test_internal_linear_algebra(ctx, tmp_path, name):
    P = problems.get(name)
    write_system(P, tmp_path)
    out = subprocess.run([str(BIN), "algebra", str(tmp_path)], capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stderr
    assert json.loads(out.stdout.strip().splitlines()[-1]) == {"dump_not_implemented": 1}
    b = P.b
    y = O.spmv(P.row_ptr, P.cols, P.vals, b)
    np.testing.assert_array_equal(f64(tmp_path, "out_mult.f64"), y)
    np.testing.assert_array_equal(f64(tmp_path, "out_copy.f64"), y)
    np.testing.assert_array_equal(f64(tmp_path, "out_axpy.f64"), O.axpy(-0.75, b, y))
    c = O.aypx(0.5, y, b)
    np.testing.assert_array_equal(f64(tmp_path, "out_aypx.f64"), c)
    np.testing.assert_array_equal(f64(tmp_path, "out_scal.f64"), 3.0 * c)
    dcol = [P.row_ptr[i] + int(np.searchsorted(P.cols[P.row_ptr[i]:P.row_ptr[i + 1]], i)) for i in range(P.n)]
    diag = np.array([P.vals[k] if k < P.row_ptr[i + 1] and P.cols[k] == i else 0.0 for i, k in enumerate(dcol)])
    np.testing.assert_array_equal(f64(tmp_path, "out_diagonal.f64"), diag)
    np.testing.assert_array_equal(f64(tmp_path, "out_reciprocal.f64"), 1.0 / diag)
    np.testing.assert_array_equal(f64(tmp_path, "out_pmult.f64"), b * (1.0 / diag))
    dot, n0, n1, n2 = f64(tmp_path, "out_scalars.f64")
    tb = ctx.info.reduction_max_blocks
    assert dot == O.dot_tree(b, b, tb)
    assert n0 == np.max(np.abs(b))
    assert n1 == pytest.approx(np.sum(np.abs(b)), rel=1e-14)
    assert n2 == np.sqrt(O.dot_tree(b, b, tb))


SOLVES = [("diffusion24", "cg", "ilu0", ""), ("diffusion24", "cg", "diag", ""), ("convdiff16", "bicgs", "ilu0", ""),
          ("poisson16", "cg", "diag", "mixed")]


@needs_bin
@pytest.mark.parametrize("name,solver,pc,mode", SOLVES)
def test_internal_linear_solver(ctx, tmp_path, name, solver, pc, mode):
    P = problems.get(name)
    write_system(P, tmp_path)
    tol, max_iter = 1e-8, 1000
    out = subprocess.run([str(BIN), "solve", str(tmp_path), solver, pc, repr(tol), str(max_iter)] +
                         ([mode] if mode else []), capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stderr
    res = json.loads(out.stdout.strip().splitlines()[-1])
    x = f64(tmp_path, "x.f64")
    assert res["ok"] == 1 and res["succeeded"] == 1 and res["error"] == 0 and res["parallel"] == 0
    assert res["solve_count"] == 1 and res["stat_iterations"] == res["last_iterations"] == res["iterations"]
    assert res["solve_time"] > 0
    assert "Last iteration number" in out.stderr  # SolverStat::print through the trace manager
    tb = ctx.info.reduction_max_blocks
    if mode == "mixed":
        o = O.mixed_solve(P.row_ptr, P.cols, P.vals, P.b, solver=solver, precond=pc, tol=tol, max_outer=20,
                          inner_tol=1e-4, inner_max_iter=max_iter, dot_mode=O.DOT_DEVICE_TREE, tree_blocks=tb,
                          jacobi_scaled=True)
        assert res["iterations"] == o.inner_iterations
        assert res["residual"] == o.true_residual
    else:
        o = O.solve(P.row_ptr, P.cols, P.vals, P.b, solver=solver, precond=pc, tol=tol, max_iter=max_iter,
                    dot_mode=O.DOT_DEVICE_TREE, tree_blocks=tb)
        assert res["iterations"] == o.iterations
        assert res["residual"] == pytest.approx(o.residual, rel=1e-12)
    np.testing.assert_array_equal(x, o.x)
