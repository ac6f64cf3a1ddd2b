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


STENCIL_SHAPED = {"poisson16", "diffusion12", "convdiff_10x11x12", "diffusion24", "grid_37x21x5"}


@pytest.mark.parametrize("schedule", ["auto", "wavefront"])
@pytest.mark.parametrize("name", ["poisson16", "diffusion12", "convdiff_10x11x12", "diffusion2d_31x9", "ragged",
                                  "diffusion24", "grid_37x21x5"])
def test_ilu0_factor_and_apply_bit_exact(ctx, name, schedule):
    P = abi.diffusion(37, 21, 5, sigma=1.0, smooth=2.0, seed=9) if name == "grid_37x21x5" else problems.get(name)
    A = ctx.matrix(P.row_ptr, P.cols, P.vals)
    pc = abi.Precond(ctx, A, "ilu0", ilu_schedule=schedule)
    expect = abi.ILU_SCHEDULE["stencil_cluster" if schedule == "auto" and name in STENCIL_SHAPED else "wavefront"]
    assert pc.info.ilu_schedule == expect
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


@pytest.mark.parametrize("schedule", ["stencil", "stencil_cluster"])
def test_ilu0_stencil_schedule_refused_for_other_matrices(ctx, schedule):
    P = problems.get("ragged")
    A = ctx.matrix(P.row_ptr, P.cols, P.vals)
    with pytest.raises(abi.AB2Error) as e:
        abi.Precond(ctx, A, "ilu0", ilu_schedule=schedule)
    assert e.value.code == abi.AB2_ERR_BAD_ARG


def test_ilu0_cluster_schedule_needs_its_buffers_in_shared_memory(ctx):
    """600 planes along z: the cluster walk's buffers exceed shared memory,
    so AUTO takes the single-CTA walk and an explicit request is refused."""
    P = abi.diffusion(20, 18, 600, sigma=1.0, smooth=2.0, seed=3)
    A = ctx.matrix(P.row_ptr, P.cols, P.vals)
    pc = abi.Precond(ctx, A, "ilu0")
    assert pc.info.ilu_schedule == abi.ILU_SCHEDULE["stencil"]
    y = rnd(P.n, 4)
    vy, vx = ctx.vector(y), ctx.vector(P.n)
    pc.apply(vy, vx)
    np.testing.assert_array_equal(vx.download(), O.ilu0_apply(P.row_ptr, P.cols, P.vals, y))
    with pytest.raises(abi.AB2Error) as e:
        abi.Precond(ctx, A, "ilu0", ilu_schedule="stencil_cluster")
    assert e.value.code == abi.AB2_ERR_BAD_ARG


def test_diag_apply(ctx):
    P = problems.get("diffusion12")
    A = ctx.matrix(P.row_ptr, P.cols, P.vals)
    pc = abi.Precond(ctx, A, "diag")
    y = rnd(P.n, 1)
    vy, vx = ctx.vector(y), ctx.vector(P.n)
    pc.apply(vy, vx)
    np.testing.assert_array_equal(vx.download(), O.inv_diag(P.row_ptr, P.cols, P.vals) * y)


@pytest.mark.parametrize("saad,lanczos", [(True, False), (True, True), (False, True)])
@pytest.mark.parametrize("name", ["poisson16", "diffusion24", "convdiff_10x11x12"])
def test_chebyshev_variants_bit_exact(ctx, name, saad, lanczos):
    """Saad's recurrence (ChebyshevPreconditioner<.., true>) and Lanczos bounds,
    against the oracle summing its dots in the device tree."""
    P = problems.get(name)
    A = ctx.matrix(P.row_ptr, P.cols, P.vals)
    pc = abi.Precond(ctx, A, "cheb", poly_factor=0.0, poly_order=3, poly_factor_max_iter=20, cheb_saad=saad,
                     cheb_lanczos=lanczos)
    tb = ctx.info.reduction_max_blocks
    x = rnd(P.n, 5)
    vx, vy = ctx.vector(x), ctx.vector(P.n)
    pc.apply(vx, vy)
    exact = O.cheb_apply(P.row_ptr, P.cols, P.vals, x, 0.0, 3, 20, dot_mode=O.DOT_DEVICE_TREE, tree_blocks=tb,
                         saad=saad, lanczos=lanczos)
    np.testing.assert_array_equal(vy.download(), exact)
    pc.apply(vx, vx)  # in place
    np.testing.assert_array_equal(vx.download(), exact)


@pytest.mark.parametrize("name,factor", [("poisson16", 0.0), ("diffusion12", 0.0), ("poisson16", 0.5),
                                         ("ragged", 0.0)])
def test_chebyshev_bounds_and_apply(ctx, name, factor):
    P = problems.get(name)
    A = ctx.matrix(P.row_ptr, P.cols, P.vals)
    pc = abi.Precond(ctx, A, "cheb", poly_factor=factor, poly_order=3, poly_factor_max_iter=12)
    tb = ctx.info.reduction_max_blocks
    # bit-exact against the oracle summing its dots in the device tree
    a, b = O.cheb_bounds(P.row_ptr, P.cols, P.vals, factor, 12, dot_mode=O.DOT_DEVICE_TREE, tree_blocks=tb)
    assert (pc.info.cheb_alpha, pc.info.cheb_beta) == (a, b)
    # and close to the sequential-dot bounds of the reference's order
    a0, b0 = O.cheb_bounds(P.row_ptr, P.cols, P.vals, factor, 12)
    assert abs(pc.info.cheb_alpha - a0) <= 1e-12 * abs(a0)
    assert abs(pc.info.cheb_beta - b0) <= 1e-12 * abs(b0)
    x = rnd(P.n, 3)
    vx, vy = ctx.vector(x), ctx.vector(P.n)
    pc.apply(vx, vy)
    exact = O.cheb_apply(P.row_ptr, P.cols, P.vals, x, factor, 3, 12, dot_mode=O.DOT_DEVICE_TREE, tree_blocks=tb)
    np.testing.assert_array_equal(vy.download(), exact)
    ref = O.cheb_apply(P.row_ptr, P.cols, P.vals, x, factor, 3, 12)
    np.testing.assert_allclose(vy.download(), ref, rtol=0, atol=1e-11 * np.max(np.abs(ref)))
    pc.apply(vx, vx)  # aliasing input/output
    np.testing.assert_array_equal(vx.download(), exact)


# The stencil sweeps one tile per CTA and in 2 x 2-tile thread-block clusters
# (tiles handing boundary values to their cluster neighbours through
# distributed shared memory), on grids whose tiles fill several clusters,
# partly filled clusters and partial tiles included.  Same bits as the
# sequential sweeps.
@pytest.mark.parametrize("schedule", ["stencil", "stencil_cluster"])
@pytest.mark.parametrize("dims", [(130, 75, 7), (40, 40, 6), (16, 100, 3), (100, 16, 3), (20, 18, 340)])
def test_ilu0_stencil_walks_bit_exact(ctx, schedule, dims):
    P = abi.diffusion(*dims, sigma=1.0, smooth=2.0, seed=5)
    A = ctx.matrix(P.row_ptr, P.cols, P.vals)
    pc = abi.Precond(ctx, A, "ilu0", ilu_schedule=schedule)
    assert pc.info.ilu_schedule == abi.ILU_SCHEDULE[schedule]
    for seed in range(2):
        y = rnd(P.n, 20 + seed)
        vy, vx = ctx.vector(y), ctx.vector(P.n)
        pc.apply(vy, vx)
        np.testing.assert_array_equal(vx.download(), O.ilu0_apply(P.row_ptr, P.cols, P.vals, y))
