"""Alien's own Krylov templates, unmodified, running on libab2.

tests/cpp/drop_in is built (tests/cpp/Makefile) from the reference's
expression/krylov/{Iteration,CG,BiCGStab,DiagPreconditioner,
ChebyshevPreconditioner,NeumannPolyPreconditioner}.h instantiated with Alien::B200::Algebra
(include/alien/b200/B200Algebra.h): the reference's CG/BiCGStab loops and
preconditioner code call the C ABI for every vector operation, SpMV and dot.
Since libab2's dots use its fixed reduction tree, the run must agree bit for
bit with the oracle summing its dots in that tree -- same iterations, same
solution -- which shows the adapter is a drop-in AlgebraT for those
templates.  Skipped when the binary was not built (no reference sources).
"""
import json
import subprocess
from pathlib import Path

import numpy as np
import pytest

from oracle import oracle as O
from tests import problems

pytestmark = pytest.mark.gpu

BIN = Path(__file__).resolve().parent / "cpp" / "_build" / "drop_in"
PC_MAP = {"diag": dict(precond="diag"), "ilu0": dict(precond="ilu0"),
          "cheb": dict(precond="cheb", poly_factor=0.0, poly_order=3, poly_factor_max_iter=20),
          "cheb_saad": dict(precond="cheb", poly_factor=0.0, poly_order=3, poly_factor_max_iter=20, cheb_saad=True),
          "neumann": dict(precond="neumann", poly_order=3),  # poly_factor: 1 / the Gershgorin bound, per matrix
          "filu0": dict(precond="filu0", filu_factor_iter=0, filu_solver_iter=3)}

CASES = [("poisson16", "cg", "diag", ""), ("poisson16", "cg", "diag", "solve2"), ("diffusion12", "cg", "ilu0", ""),
         ("diffusion24", "cg", "cheb_saad", ""), ("poisson16", "cg", "cheb", ""),
         ("convdiff_10x11x12", "bicgs", "ilu0", ""), ("convdiff_10x11x12", "bicgs", "diag", "solve2"),
         ("ragged", "bicgs", "diag", ""), ("diffusion2d_31x9", "bicgs", "ilu0", ""),
         ("poisson16", "cg", "neumann", ""), ("poisson16", "bicgs", "filu0", ""),
         ("convdiff_10x11x12", "bicgs", "filu0", "solve2")]


@pytest.mark.skipif(not BIN.exists(), reason="tests/cpp/_build/drop_in not built (reference sources absent)")
@pytest.mark.parametrize("name,solver,pc,mode", CASES)
def test_reference_templates_on_b200_algebra(ctx, tmp_path, name, solver, pc, mode):
    P = problems.get(name)
    P.row_ptr.astype(np.int32).tofile(tmp_path / "rp.i32")
    P.cols.astype(np.int32).tofile(tmp_path / "ci.i32")
    P.vals.astype(np.float64).tofile(tmp_path / "v.f64")
    P.b.astype(np.float64).tofile(tmp_path / "b.f64")
    kw = dict(PC_MAP[pc])
    if pc == "neumann":
        kw["poly_factor"] = 1.0 / float(np.add.reduceat(np.abs(P.vals), P.row_ptr[:-1]).max())
        (tmp_path / "omega.txt").write_text(repr(kw["poly_factor"]))
    tol, max_iter = 1e-8, 400
    out = subprocess.run([str(BIN), str(tmp_path), solver, pc, repr(tol), str(max_iter)] + ([mode] if mode else []),
                         capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stderr
    res = json.loads(out.stdout.strip().splitlines()[-1])
    x = np.fromfile(tmp_path / "x.f64", dtype=np.float64)
    o = O.solve(P.row_ptr, P.cols, P.vals, P.b, solver=solver, tol=tol, max_iter=max_iter,
                dot_mode=O.DOT_DEVICE_TREE, tree_blocks=ctx.info.reduction_max_blocks, **kw)
    assert res["iterations"] == o.iterations and res["converged"] == o.converged
    assert res["breakdown"] == o.breakdown
    np.testing.assert_array_equal(x, o.x)
    assert res["gpu_launches"] > 2 * res["iterations"]
