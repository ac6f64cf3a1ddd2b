"""Mixed-precision solver (FP32 Krylov inside FP64 refinement) vs the oracle.

No counterpart in the reference, so parity is against this repo's
restatement (oracle/ab2_oracle.cpp orc_mixed_solve: the reference templates'
arithmetic instantiated in float, FP64 residual and update), with every dot
summed in libab2's reduction tree: same refinement steps, same FP32 inner
iteration counts, same true-residual history and the same solution bits.
That pins the FP32 SpMV (CSR and sliced ELL), the FP32 preconditioners (Diag,
ILU(0) on both schedules, Chebyshev), the FP32 dots and scalar recurrences and
the FP64 refinement kernels.  Each result also states its error against an
FP64 solution (the oracle's plain FP64 solve to 1e-13).
"""
import numpy as np
import pytest

from alien_b200 import abi
from oracle import oracle as O
from tests import problems

pytestmark = pytest.mark.gpu

F32 = abi.FMT_CSR | abi.FMT_ELL | abi.FMT_F32

CASES = [
    ("poisson16", "cg", "diag", {}),
    ("poisson16", "cg", "ilu0", {}),
    ("diffusion12", "cg", "ilu0", {}),
    ("diffusion24", "cg", "cheb", dict(cheb_saad=True)),
    ("diffusion24", "cg", "cheb", dict(cheb_saad=True, cheb_lanczos=True)),
    ("convdiff_10x11x12", "bicgs", "ilu0", {}),
    ("convdiff_10x11x12", "bicgs", "diag", {}),
    ("convdiff16", "bicgs", "ilu0", {}),
    ("diffusion2d_31x9", "bicgs", "ilu0", {}),  # wavefront ILU(0) schedule in FP32
    ("ragged", "bicgs", "diag", {}),
    ("ragged", "cg", "none", {}),
]


def fp64_solution(P, solver):
    r = O.solve(P.row_ptr, P.cols, P.vals, P.b, solver=solver, precond="ilu0", tol=1e-13, max_iter=5000)
    return r.x


@pytest.mark.parametrize("use_graph", [True, False])
@pytest.mark.parametrize("name,solver,pc,extra", CASES)
def test_mixed_bit_exact(ctx, name, solver, pc, extra, use_graph):
    P = problems.get(name)
    kw = dict(solver=solver, precond=pc, tol=1e-10, max_outer=10, inner_tol=1e-4, inner_max_iter=500, **extra)
    A = ctx.matrix(P.row_ptr, P.cols, P.vals, F32)
    M = abi.Mixed(ctx, A, use_graph=use_graph, **kw)
    b, x = ctx.vector(P.b), ctx.vector(P.n)
    st = M.solve(b, x)
    xs = x.download()
    o = O.mixed_solve(P.row_ptr, P.cols, P.vals, P.b, dot_mode=O.DOT_DEVICE_TREE,
                      tree_blocks=ctx.info.reduction_max_blocks, **kw)
    assert (st.succeeded, st.outer_iterations, st.inner_iterations) == (o.succeeded, o.outer_iterations,
                                                                       o.inner_iterations)
    np.testing.assert_array_equal(M.history(), o.history)
    np.testing.assert_array_equal(xs, o.x)
    assert st.succeeded and st.true_residual < 1e-10
    # error against an FP64 solution (plain FP64 Krylov to 1e-13)
    x64 = fp64_solution(P, solver)
    assert np.linalg.norm(xs - x64) / np.linalg.norm(x64) < 1e-8


def test_mixed_needs_fp32_values(ctx):
    P = problems.get("poisson16")
    A = ctx.matrix(P.row_ptr, P.cols, P.vals)  # no FMT_F32
    with pytest.raises(abi.AB2Error) as e:
        abi.Mixed(ctx, A, precond="diag")
    assert e.value.code == abi.AB2_ERR_BAD_ARG


def test_mixed_stops_without_success(ctx):
    """max_outer reached: AB2_ERR_NOT_CONVERGED, history has max_outer + 1 entries."""
    P = problems.get("diffusion12")
    A = ctx.matrix(P.row_ptr, P.cols, P.vals, F32)
    M = abi.Mixed(ctx, A, precond="diag", tol=1e-14, max_outer=1, inner_tol=1e-3)
    st = M.solve(ctx.vector(P.b), ctx.vector(P.n))
    assert not st.succeeded and st.error == abi.AB2_ERR_NOT_CONVERGED
    assert st.outer_iterations == 1 and M.history().size == 2
    assert M.history()[1] < M.history()[0]


def test_mixed_null_rhs_and_repeat(ctx):
    P = problems.get("poisson16")
    A = ctx.matrix(P.row_ptr, P.cols, P.vals, F32)
    M = abi.Mixed(ctx, A, precond="ilu0", tol=1e-9)
    st = M.solve(ctx.vector(P.n), ctx.vector(P.n))
    assert st.succeeded and st.outer_iterations == 0
    xs = []
    for _ in range(2):  # the same object solves again from scratch
        x = ctx.vector(P.n)
        st = M.solve(ctx.vector(P.b), x)
        assert st.succeeded
        xs.append(x.download())
    np.testing.assert_array_equal(xs[0], xs[1])
