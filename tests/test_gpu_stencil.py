"""7-point bands (AB2_FMT_STENCIL) and the mixed solver's scaled Jacobi form.

A matrix created with AB2_FMT_STENCIL keeps its values as bands without
column indices when its profile is a 3-D 7-point stencil in lexicographic
order (4 bands when the values are bit-for-bit symmetric, else 7); other
profiles silently keep none.  The band SpMV sums a row's terms in the CSR
column order and skips neighbours outside the grid, so it must equal the
oracle's row-sequential sum bit for bit -- alone, inside every solver (AUTO
picks the bands) and in FP32 inside the mixed solver.  The scaled Jacobi
form has no reference counterpart: it is checked bit for bit against the
oracle's restatement (orc_mixed_solve with jacobi_scaled).
"""
import numpy as np
import pytest

from alien_b200 import abi
from oracle import oracle as O
from tests import problems

pytestmark = pytest.mark.gpu

BANDS = abi.FMT_CSR | abi.FMT_ELL | abi.FMT_F32 | abi.FMT_STENCIL

DETECT = [("poisson16", 4), ("diffusion12", 4), ("diffusion24", 4), ("convdiff_10x11x12", 7), ("convdiff16", 7),
          ("diffusion2d_31x9", 0), ("ragged", 0), ("longrow", 0)]


def rnd(n, seed):
    return np.random.default_rng(seed).uniform(-1, 1, n)


@pytest.mark.parametrize("name,bands", DETECT)
def test_detection_and_spmv_bit_exact(ctx, name, bands):
    P = problems.get(name)
    A = ctx.matrix(P.row_ptr, P.cols, P.vals, BANDS)
    info = A.info
    assert info.stencil_bands == bands
    assert bool(info.formats & abi.FMT_STENCIL) == (bands > 0)
    if bands:
        assert (info.stencil_nx, info.stencil_ny, info.stencil_nz) == tuple(P.shape)
    x = rnd(P.n, 1)
    exp = O.spmv(P.row_ptr, P.cols, P.vals, x)
    vx, vy = ctx.vector(x), ctx.vector(P.n)
    for variant in ((abi.SPMV_AUTO, abi.SPMV_STENCIL) if bands else (abi.SPMV_AUTO,)):
        ctx.mult(A, vx, vy, variant)
        np.testing.assert_array_equal(vy.download(), exp)
    if not bands:
        with pytest.raises(abi.AB2Error):
            ctx.mult(A, vx, vy, abi.SPMV_STENCIL)
    A.close()


def test_neighbours_outside_the_grid_are_skipped(ctx):
    """x = inf on every cell with i == 0: rows with i == nx - 1 have their
    +x neighbour in the next grid line's first cell, which is not in the row;
    adding it as 0 * inf would give NaN.  The result must be the oracle's."""
    P = problems.get("diffusion12")
    nx = P.shape[0]
    A = ctx.matrix(P.row_ptr, P.cols, P.vals, BANDS)
    x = rnd(P.n, 2)
    x[np.arange(P.n) % nx == 0] = np.inf
    vx, vy = ctx.vector(x), ctx.vector(P.n)
    ctx.mult(A, vx, vy, abi.SPMV_STENCIL)
    got = vy.download()
    exp = O.spmv(P.row_ptr, P.cols, P.vals, x)
    np.testing.assert_array_equal(got, exp)
    assert np.all(np.isfinite(got[np.arange(P.n) % nx == nx - 1]))
    A.close()


def test_update_values_redecides_symmetry(ctx):
    P = problems.get("poisson16")
    A = ctx.matrix(P.row_ptr, P.cols, P.vals, BANDS)
    assert A.info.stencil_bands == 4
    v = P.vals.copy()
    row = 1000
    k = int(np.nonzero(P.cols[P.row_ptr[row]:P.row_ptr[row + 1]] == row + 1)[0][0]) + P.row_ptr[row]
    v[k] = -0.75  # the pair (row, row+1) is no longer symmetric
    A.update_values(v)
    assert A.info.stencil_bands == 7
    x = rnd(P.n, 3)
    vx, vy = ctx.vector(x), ctx.vector(P.n)
    ctx.mult(A, vx, vy)
    np.testing.assert_array_equal(vy.download(), O.spmv(P.row_ptr, P.cols, v, x))
    A.update_values(P.vals)
    assert A.info.stencil_bands == 4
    ctx.mult(A, vx, vy)
    np.testing.assert_array_equal(vy.download(), O.spmv(P.row_ptr, P.cols, P.vals, x))
    A.close()


SOLVES = [
    ("diffusion24", "cg", "diag", {}),
    ("diffusion24", "cg", "ilu0", {}),
    ("diffusion24", "cg", "none", {}),
    ("poisson16", "cg", "cheb", dict(cheb_saad=True, poly_factor_max_iter=10)),
    ("convdiff16", "bicgs", "ilu0", {}),
    ("convdiff_10x11x12", "bicgs", "diag", {}),
]


@pytest.mark.parametrize("use_graph", [True, False])
@pytest.mark.parametrize("name,solver,pc,extra", SOLVES)
def test_fp64_solves_on_bands_bit_exact(ctx, name, solver, pc, extra, use_graph):
    P = problems.get(name)
    A = ctx.matrix(P.row_ptr, P.cols, P.vals, BANDS)
    assert A.info.stencil_bands in (4, 7)
    kw = dict(solver=solver, precond=pc, tol=1e-8, max_iter=1000, **extra)
    S = abi.Solver(ctx, A, use_graph=use_graph, **kw)
    b, x = ctx.vector(P.b), ctx.vector(P.n)
    st = S.solve(b, x)
    t = O.solve(P.row_ptr, P.cols, P.vals, P.b, dot_mode=O.DOT_DEVICE_TREE,
                tree_blocks=ctx.info.reduction_max_blocks, **kw)
    assert (st.iterations, st.succeeded) == (t.iterations, t.converged)
    np.testing.assert_array_equal(S.history(), t.history)
    np.testing.assert_array_equal(x.download(), t.x)
    S.close()
    A.close()


MIXED = [
    ("diffusion24", "cg", "diag", "auto", True),
    ("diffusion24", "cg", "diag", "plain", False),
    ("poisson16", "cg", "diag", "scaled", True),
    ("diffusion_10x11x12", "cg", "diag", "auto", True),
    ("diffusion_20x6x9", "cg", "diag", "scaled", True),
    ("diffusion_20x6x9", "cg", "diag", "plain", False),
    ("diffusion_80x72x64", "cg", "diag", "auto", True),
    ("diffusion12", "cg", "ilu0", "auto", False),
    ("convdiff16", "bicgs", "ilu0", "auto", False),
    ("convdiff_10x11x12", "bicgs", "diag", "auto", False),
]


@pytest.mark.parametrize("use_graph", [True, False])
@pytest.mark.parametrize("name,solver,pc,form,scaled", MIXED)
def test_mixed_on_bands_bit_exact(ctx, name, solver, pc, form, scaled, use_graph):
    P = problems.get(name)
    A = ctx.matrix(P.row_ptr, P.cols, P.vals, BANDS)
    kw = dict(solver=solver, precond=pc, tol=1e-10, max_outer=10, inner_tol=1e-4, inner_max_iter=500)
    M = abi.Mixed(ctx, A, use_graph=use_graph, jacobi_form=form, **kw)
    b, x = ctx.vector(P.b), ctx.vector(P.n)
    st = M.solve(b, x)
    assert st.jacobi_scaled == scaled
    o = O.mixed_solve(P.row_ptr, P.cols, P.vals, P.b, dot_mode=O.DOT_DEVICE_TREE,
                      tree_blocks=ctx.info.reduction_max_blocks, jacobi_scaled=scaled, **kw)
    assert (st.succeeded, st.outer_iterations, st.inner_iterations) == (o.succeeded, o.outer_iterations,
                                                                       o.inner_iterations)
    np.testing.assert_array_equal(M.history(), o.history)
    np.testing.assert_array_equal(x.download(), o.x)
    assert st.succeeded and st.true_residual < 1e-10
    M.close()
    A.close()


def test_scaled_form_needs_symmetric_bands(ctx):
    for name, fmt in (("convdiff16", BANDS), ("diffusion12", abi.FMT_CSR | abi.FMT_ELL | abi.FMT_F32)):
        P = problems.get(name)
        A = ctx.matrix(P.row_ptr, P.cols, P.vals, fmt)
        with pytest.raises(abi.AB2Error) as e:
            abi.Mixed(ctx, A, solver="cg", precond="diag", jacobi_form="scaled")
        assert e.value.code == abi.AB2_ERR_BAD_ARG
        A.close()


def test_explicit_zeros_in_the_profile_stay_terms(ctx):
    """Entries stored with the value 0 are part of the row (as in the CSR
    sum): 0 * inf gives NaN in the band SpMV exactly where the row-sequential
    sum gives it."""
    P = problems.get("poisson16")
    v = P.vals.copy()
    rows = [100, 777, 2048]
    for r in rows:  # zero the (r, r+1) / (r+1, r) pair: still symmetric
        a = P.row_ptr[r] + int(np.nonzero(P.cols[P.row_ptr[r]:P.row_ptr[r + 1]] == r + 1)[0][0])
        b = P.row_ptr[r + 1] + int(np.nonzero(P.cols[P.row_ptr[r + 1]:P.row_ptr[r + 2]] == r)[0][0])
        v[a] = v[b] = 0.0
    A = ctx.matrix(P.row_ptr, P.cols, v, BANDS)
    assert A.info.stencil_bands == 4
    x = rnd(P.n, 9)
    x[[r + 1 for r in rows]] = np.inf
    vx, vy = ctx.vector(x), ctx.vector(P.n)
    ctx.mult(A, vx, vy, abi.SPMV_STENCIL)
    got = vy.download()
    exp = O.spmv(P.row_ptr, P.cols, v, x)
    np.testing.assert_array_equal(got, exp)
    assert np.all(np.isnan(got[rows]))
    A.close()
