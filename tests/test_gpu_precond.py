"""Preconditioners on the GPU vs the CPU oracle.

ILU(0): factor and applications bit-identical to the reference's sequential
LUFactorisationAlgo (same per-row arithmetic, wavefront-parallel order).
Chebyshev: the power-method bounds use device dot products (fixed tree), so
bounds and applications agree to rounding only (1e-12 relative).
"""
import numpy as np
import pytest

from alien_b200 import abi
from oracle import oracle as O
from tests import problems

pytestmark = pytest.mark.gpu


def rnd(n, seed):
    return np.random.default_rng(seed).uniform(-1, 1, n)


@pytest.mark.parametrize("name", ["poisson16", "diffusion12", "convdiff_10x11x12", "diffusion2d_31x9", "ragged",
                                  "diffusion24"])
def test_ilu0_factor_and_apply_bit_exact(ctx, name):
    P = problems.get(name)
    A = ctx.matrix(P.row_ptr, P.cols, P.vals)
    pc = abi.Precond(ctx, A, "ilu0")
    np.testing.assert_array_equal(pc.ilu0_values(), O.ilu0_factor(P.row_ptr, P.cols, P.vals))
    for seed in range(3):  # repeated applications (sweep state must reset itself)
        y = rnd(P.n, seed)
        vy, vx = ctx.vector(y), ctx.vector(P.n)
        pc.apply(vy, vx)
        np.testing.assert_array_equal(vx.download(), O.ilu0_apply(P.row_ptr, P.cols, P.vals, y))
    # in place: x and y the same vector
    y = rnd(P.n, 9)
    v = ctx.vector(y)
    pc.apply(v, v)
    np.testing.assert_array_equal(v.download(), O.ilu0_apply(P.row_ptr, P.cols, P.vals, y))
    info = pc.info
    assert info.ilu_levels_lower >= 1 and info.ilu_levels_upper >= 1
    if name == "poisson16":
        assert info.ilu_levels_lower == 3 * 16 - 2


def test_diag_apply(ctx):
    P = problems.get("diffusion12")
    A = ctx.matrix(P.row_ptr, P.cols, P.vals)
    pc = abi.Precond(ctx, A, "diag")
    y = rnd(P.n, 1)
    vy, vx = ctx.vector(y), ctx.vector(P.n)
    pc.apply(vy, vx)
    np.testing.assert_array_equal(vx.download(), O.inv_diag(P.row_ptr, P.cols, P.vals) * y)


@pytest.mark.parametrize("name,factor", [("poisson16", 0.0), ("diffusion12", 0.0), ("poisson16", 0.5),
                                         ("ragged", 0.0)])
def test_chebyshev_bounds_and_apply(ctx, name, factor):
    P = problems.get(name)
    A = ctx.matrix(P.row_ptr, P.cols, P.vals)
    pc = abi.Precond(ctx, A, "cheb", poly_factor=factor, poly_order=3, poly_factor_max_iter=12)
    a, b = O.cheb_bounds(P.row_ptr, P.cols, P.vals, factor, 12)
    assert abs(pc.info.cheb_alpha - a) <= 1e-12 * abs(a)
    assert abs(pc.info.cheb_beta - b) <= 1e-12 * abs(b)
    x = rnd(P.n, 3)
    vx, vy = ctx.vector(x), ctx.vector(P.n)
    pc.apply(vx, vy)
    ref = O.cheb_apply(P.row_ptr, P.cols, P.vals, x, factor, 3, 12)
    np.testing.assert_allclose(vy.download(), ref, rtol=0, atol=1e-11 * np.max(np.abs(ref)))
    pc.apply(vx, vx)  # aliasing input/output
    np.testing.assert_allclose(vx.download(), ref, rtol=0, atol=1e-11 * np.max(np.abs(ref)))
