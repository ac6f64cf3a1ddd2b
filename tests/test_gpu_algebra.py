"""GPU algebra through the C ABI vs the CPU oracle.

SpMV, L/U products, inverse diagonal and the BLAS-1 updates round exactly as
the reference's sequential loops, so they must match the oracle bit for bit;
dot products use a fixed reduction tree and must agree to 1e-14 (relative to
sum |x_i y_i|) and be bit-reproducible run to run.
"""
import numpy as np
import pytest

from alien_b200 import abi
from oracle import oracle as O
from tests import problems

pytestmark = pytest.mark.gpu

MATRICES = ["poisson16", "diffusion12", "convdiff_10x11x12", "diffusion2d_31x9", "ragged", "longrow"]
VARIANTS = [abi.SPMV_CSR_SCALAR, abi.SPMV_CSR_STAGED, abi.SPMV_ELL]


def rnd(n, seed):
    return np.random.default_rng(seed).uniform(-1, 1, n)


@pytest.mark.parametrize("name", MATRICES)
@pytest.mark.parametrize("variant", VARIANTS)
def test_spmv_bit_exact(ctx, name, variant):
    P = problems.get(name)
    A = ctx.matrix(P.row_ptr, P.cols, P.vals, abi.FMT_CSR | abi.FMT_ELL)
    x = rnd(P.n, 1)
    vx, vy = ctx.vector(x), ctx.vector(P.n)
    ctx.mult(A, vx, vy, variant)
    np.testing.assert_array_equal(vy.download(), O.spmv(P.row_ptr, P.cols, P.vals, x))


@pytest.mark.parametrize("name", MATRICES + ["diffusion64", "wide12", "wide24", "wide200", "wide1000"])
def test_spmv_warp_per_row(ctx, name):
    """The grouped-lane variant splits a row across 4, 8, 16 or 32 lanes (by
    mean row length; the wide* matrices reach every width) and adds their
    partial sums in a shuffle tree: not the sequential order, so it is held to
    1e-13 of sum |a_ij x_j| per row, and must be bit-reproducible."""
    P = problems.get(name)
    A = ctx.matrix(P.row_ptr, P.cols, P.vals, abi.FMT_CSR)
    x = rnd(P.n, 4)
    vx, vy = ctx.vector(x), ctx.vector(P.n)
    ctx.mult(A, vx, vy, abi.SPMV_CSR_VECTOR)
    got = vy.download()
    exp = O.spmv(P.row_ptr, P.cols, P.vals, x)
    scale = O.spmv(P.row_ptr, P.cols, np.abs(P.vals), np.abs(x))
    assert np.all(np.abs(got - exp) <= 1e-13 * scale)
    ctx.mult(A, vx, vy, abi.SPMV_CSR_VECTOR)
    np.testing.assert_array_equal(vy.download(), got)
    A.close()


@pytest.mark.parametrize("name", ["diffusion12", "ragged"])
def test_lu_products_invdiag(ctx, name):
    P = problems.get(name)
    A = ctx.matrix(P.row_ptr, P.cols, P.vals)
    x, y0 = rnd(P.n, 2), rnd(P.n, 3)
    vx = ctx.vector(x)
    for lower in (True, False):
        vy = ctx.vector(y0)
        (ctx.addLMult if lower else ctx.addUMult)(-0.7, A, vx, vy)
        np.testing.assert_array_equal(vy.download(), O.add_lu_mult(P.row_ptr, P.cols, P.vals, -0.7, x, y0, lower))
    d = ctx.vector(P.n)
    ctx.computeInvDiag(A, d)
    inv = O.inv_diag(P.row_ptr, P.cols, P.vals)
    np.testing.assert_array_equal(d.download(), inv)
    diag = np.array([P.vals[P.row_ptr[i] + np.searchsorted(P.cols[P.row_ptr[i]:P.row_ptr[i + 1]], i)]
                     for i in range(P.n)])
    y = ctx.vector(y0)
    ctx.multInvDiag(A, y)  # y / a_ii (SimpleCSRMatrixMultT.h:478-492)
    np.testing.assert_array_equal(y.download(), y0 / diag)
    ctx.diagonal(A, d)
    np.testing.assert_array_equal(d.download(), diag)


def test_blas1_bit_exact(ctx):
    n = 100003
    x, y = rnd(n, 4), rnd(n, 5)
    vx, vy, vw = ctx.vector(x), ctx.vector(y), ctx.vector(n)
    ctx.axpy(0.37, vx, vy)  # y = fma(a, x, y), as CBLAS daxpy
    exp_axpy = O.axpy(0.37, x, y)
    np.testing.assert_array_equal(vy.download(), exp_axpy)
    ctx.aypx(-1.5, vy, vx)  # y = a y + x
    exp_aypx = O.aypx(-1.5, exp_axpy, x)
    np.testing.assert_array_equal(vy.download(), exp_aypx)
    ctx.scal(3.0, vy)
    np.testing.assert_array_equal(vy.download(), 3.0 * exp_aypx)
    ctx.pointwiseMult(vx, vy, vw)
    np.testing.assert_array_equal(vw.download(), x * (3.0 * exp_aypx))
    ctx.pointwiseMult(vx, vw, vw)  # aliasing output, as DiagPreconditioner uses it
    np.testing.assert_array_equal(vw.download(), x * (x * (3.0 * exp_aypx)))
    ctx.copy(vx, vw)
    np.testing.assert_array_equal(vw.download(), x)
    ctx.reciprocal(vw)
    np.testing.assert_array_equal(vw.download(), 1.0 / x)
    ctx.assign(vw, 2.5)
    np.testing.assert_array_equal(vw.download(), np.full(n, 2.5))


@pytest.mark.parametrize("n", [0, 1, 31, 32, 33, 1000, 1 << 20, 3_000_017])
def test_dot_norms(ctx, n):
    import math

    x, y = rnd(n, 6), rnd(n, 7)
    vx, vy = ctx.vector(x), ctx.vector(y)
    d = ctx.dot(vx, vy)
    # The device tree's error is ~log2(n) eps sum|x_i y_i|; compare with the
    # exactly rounded sum (the sequential oracle carries ~n eps itself).
    scale = max(float(np.sum(np.abs(x * y))), 1e-300)
    exact = math.fsum(np.fma(x, y, 0.0) if hasattr(np, "fma") else x * y)
    assert abs(d - exact) <= 1e-14 * scale
    assert abs(d - O.dot(x, y)) <= (1e-14 + n * 2.3e-16) * scale
    assert ctx.dot(vx, vy) == d  # deterministic tree
    assert d == O.dot_tree(x, y, ctx.info.reduction_max_blocks)  # and exactly the documented one
    xx = math.fsum(x * x)
    assert abs(ctx.norm2(vx) - math.sqrt(xx)) <= 1e-14 * max(math.sqrt(xx), 1e-300)
    assert abs(ctx.norm1(vx) - math.fsum(np.abs(x))) <= 1e-14 * max(math.fsum(np.abs(x)), 1e-300)
    assert ctx.norm0(vx) == (np.max(np.abs(x)) if n else 0.0)


def test_dot_future(ctx):
    import ctypes as C
    L = abi.lib()
    x, y = rnd(5000, 8), rnd(5000, 9)
    vx, vy = ctx.vector(x), ctx.vector(y)
    s = C.c_void_p()
    ctx.check(L.ab2_scalar_create(ctx.h, C.byref(s)))
    ctx.check(L.ab2_dot_async(ctx.h, vx.h, vy.h, s))
    out = C.c_double()
    ctx.check(L.ab2_scalar_get(ctx.h, s, C.byref(out)))
    assert out.value == ctx.dot(vx, vy)
    L.ab2_scalar_destroy(s)


def test_testmvexpr_known_answers_on_gpu(ctx):
    """Alien's own algebra KATs (src/refsemantic/tests/TestMVExpr.cc:105-167), on the device."""
    rp, ci, v = problems.laplacian_1d(10)
    A = ctx.matrix(rp, ci, v)
    lam, n = 0.5, 10
    x, y, r = ctx.vector(np.ones(n)), ctx.vector(n), ctx.vector(n)
    assert ctx.norm2(x) == np.sqrt(10)
    ctx.copy(x, y)
    ctx.scal(lam, y)
    assert ctx.norm2(y) == np.sqrt(n * 0.25)
    ctx.mult(A, x, y)
    assert ctx.norm2(y) == np.sqrt(2)
    ctx.mult(A, x, r)
    ctx.scal(-1.0, r)
    ctx.axpy(1.0, y, r)
    assert ctx.norm2(r) == 0.0
    ctx.axpy(lam, x, y)
    assert ctx.norm2(y) == np.sqrt(2 * 1.5 * 1.5 + (n - 2) * 0.25)
    lx = ctx.vector(np.full(n, lam))
    ctx.mult(A, lx, y)
    assert ctx.norm2(y) == np.sqrt(0.5)
    y.upload(np.arange(n, dtype=np.float64))
    assert ctx.dot(x, y) == 45
    assert ctx.dot(lx, y) == 22.5
    ay = ctx.vector(n)
    ctx.mult(A, y, ay)
    assert ctx.dot(x, ay) == 9


def test_invalid_inputs_rejected(ctx):
    rp = np.array([0, 2, 3], dtype=np.int32)
    with pytest.raises(abi.AB2Error) as e:
        ctx.matrix(rp, np.array([0, 5, 1], dtype=np.int32), np.ones(3))  # column out of range
    assert e.value.code == abi.AB2_ERR_BAD_ARG
    with pytest.raises(abi.AB2Error):
        ctx.matrix(rp, np.array([1, 0, 1], dtype=np.int32), np.ones(3))  # unsorted row
    P = problems.get("poisson16")
    A = ctx.matrix(P.row_ptr, P.cols, P.vals)
    with pytest.raises(abi.AB2Error):
        ctx.mult(A, ctx.vector(P.n), ctx.vector(P.n - 1))
    v = ctx.vector(P.n)
    with pytest.raises(abi.AB2Error):
        ctx.mult(A, v, v)  # y must not alias x


def test_empty_matrix(ctx):
    A = ctx.matrix(np.zeros(1, np.int32), np.zeros(0, np.int32), np.zeros(0))
    x, y = ctx.vector(0), ctx.vector(0)
    ctx.mult(A, x, y)
    assert ctx.dot(x, y) == 0.0


def test_update_values(ctx):
    P = problems.get("diffusion12")
    A = ctx.matrix(P.row_ptr, P.cols, P.vals)
    v2 = P.vals * 1.5
    A.update_values(v2)
    x = rnd(P.n, 10)
    vx, vy = ctx.vector(x), ctx.vector(P.n)
    ctx.mult(A, vx, vy, abi.SPMV_ELL)
    np.testing.assert_array_equal(vy.download(), O.spmv(P.row_ptr, P.cols, v2, x))
