"""Failure detection on the GPU without a fault.

Every device-side wait in libab2 (the sentinel polling of the ILU(0) sweeps,
the mbarrier waits of the learned preconditioner's grid layer) is bounded by
a clock budget and an error flag.  Here one thread waits on a word that
nothing writes -- a producer that is gone -- or on an mbarrier phase that
nothing completes: the wait must give up by itself, set the flag the host
reads, and leave the context usable.  (Host-side
failures -- a rank that never reaches a collective -- are covered in
test_gpu_dist.py and test_dist.py.)
"""
import numpy as np
import pytest

from alien_b200 import abi

pytestmark = pytest.mark.gpu


def test_bounded_wait_gives_up_and_context_stays_usable(ctx):
    expired, seconds = ctx.selftest_bounded_wait()
    assert expired
    assert 0.5 < seconds < 30.0  # the budget: 4e9 cycles, ~2 s at full clock
    v = ctx.vector(np.arange(1000, dtype=np.float64))
    assert ctx.dot(v, v) == float(np.dot(np.arange(1000.0), np.arange(1000.0)))
    P = abi.poisson(8, 8, 8, seed=0)
    A = ctx.matrix(P.row_ptr, P.cols, P.vals)
    S = abi.Solver(ctx, A, solver="cg", precond="ilu0", tol=1e-8, max_iter=200)
    st = S.solve(ctx.vector(P.b), ctx.vector(P.n))
    assert st.succeeded and st.error == 0
    S.close()
    A.close()


def test_mbarrier_wait_gives_up_and_context_stays_usable(ctx):
    expired, seconds = ctx.selftest_mbarrier_wait()
    assert expired
    assert 0.5 < seconds < 30.0
    # the grid layer of the learned preconditioner still runs on this context
    from oracle import gnn_oracle as G

    P = abi.diffusion(12, 11, 10, sigma=1.5, smooth=2.0, seed=4)
    A = ctx.matrix(P.row_ptr, P.cols, P.vals)
    net = abi.Gnn(ctx, G.init_params(2).flat().astype(np.float32))
    net.bind(A)
    assert net.layer == "grid"
    z = ctx.vector(P.n)
    net.apply(ctx.vector(np.ones(P.n)), z)
    assert np.all(np.isfinite(z.download()))
    net.close()
    A.close()


def _tridiag(n, diag0):
    rp, ci, vv = [0], [], []
    for i in range(n):
        for j, v in ((i - 1, -1.0), (i, 2.0 if i else diag0), (i + 1, -1.0)):
            if 0 <= j < n:
                ci.append(j)
                vv.append(v)
        rp.append(len(ci))
    return np.asarray(rp, np.int32), np.asarray(ci, np.int32), np.asarray(vv)


def _gpu_solve(ctx, rp, ci, vv, b, **kw):
    A = ctx.matrix(rp, ci, vv)
    x = ctx.vector(rp.size - 1)
    S = abi.Solver(ctx, A, **kw)
    st = S.solve(ctx.vector(b), x)
    out = (st, x.download(), S.history())
    S.close()
    A.close()
    return out


@pytest.mark.parametrize("solver", ["cg", "bicgs"])
def test_zero_pivot_in_ilu0_input_matches_reference_arithmetic(ctx, solver):
    """a_00 = 0: the factorisation divides by zero (ILU0Preconditioner.h has
    no pivot check), infinities and NaNs flow through the solve, the stop
    test never passes; the GPU does exactly what the reference's arithmetic
    does (same iterations, same NaN/inf pattern), reported as not converged."""
    from oracle import oracle as O

    rp, ci, vv = _tridiag(50, 0.0)
    b = np.ones(50)
    st, x, h = _gpu_solve(ctx, rp, ci, vv, b, solver=solver, precond="ilu0", tol=1e-8, max_iter=20)
    o = O.solve(rp, ci, vv, b, solver=solver, precond="ilu0", tol=1e-8, max_iter=20, dot_mode=O.DOT_DEVICE_TREE,
                tree_blocks=ctx.info.reduction_max_blocks)
    assert not np.isfinite(O.ilu0_factor(rp, ci, vv)).all()
    assert (st.iterations, st.succeeded, st.breakdown) == (o.iterations, o.converged, o.breakdown)
    assert not st.succeeded
    np.testing.assert_array_equal(x, o.x)
    np.testing.assert_array_equal(h, o.history)


def test_nan_in_right_hand_side(ctx):
    """A NaN in b: b.b is NaN, so is the criterion; no stop test passes and the
    solve ends at max_iter, not converged, as the reference's Iteration does."""
    from oracle import oracle as O

    rp, ci, vv = _tridiag(40, 2.0)
    b = np.ones(40)
    b[7] = np.nan
    st, x, h = _gpu_solve(ctx, rp, ci, vv, b, solver="cg", precond="diag", tol=1e-8, max_iter=15)
    o = O.solve(rp, ci, vv, b, solver="cg", precond="diag", tol=1e-8, max_iter=15, dot_mode=O.DOT_DEVICE_TREE,
                tree_blocks=ctx.info.reduction_max_blocks)
    assert (st.iterations, st.succeeded) == (o.iterations, o.converged) == (15, False)
    np.testing.assert_array_equal(x, o.x)


def test_device_allocation_failures_unwind_cleanly():
    """Host-side injection: the n-th device allocation fails, for every n
    along matrix creation (CSR + ELL + FP32), ILU(0) set-up, solver set-up and
    solve.  Each call returns AB2_ERR_OOM without crashing or leaving the
    context unusable: the same context then solves normally."""
    from tests import problems

    P = problems.get("diffusion12")
    c = abi.Context(0)
    ref = None
    nth, failures = 1, 0
    while True:
        c.inject_alloc_failure(nth)
        try:
            A = c.matrix(P.row_ptr, P.cols, P.vals, abi.FMT_CSR | abi.FMT_ELL | abi.FMT_F32)
            S = abi.Solver(c, A, solver="cg", precond="ilu0", tol=1e-8, max_iter=200)
            x = c.vector(P.n)
            st = S.solve(c.vector(P.b), x)
            S.close()
            A.close()
            done = True
        except abi.AB2Error as e:
            assert e.code == abi.AB2_ERR_OOM, e
            failures += 1
            done = False
        c.inject_alloc_failure(0)
        A2 = c.matrix(P.row_ptr, P.cols, P.vals)
        S2 = abi.Solver(c, A2, solver="cg", precond="ilu0", tol=1e-8, max_iter=200)
        x2 = c.vector(P.n)
        st2 = S2.solve(c.vector(P.b), x2)
        assert st2.succeeded
        if ref is None:
            ref = x2.download()
        np.testing.assert_array_equal(x2.download(), ref)
        S2.close()
        A2.close()
        if done:
            assert st.succeeded
            break
        nth += 1
        assert nth < 200
    assert failures >= 10  # every allocation of the chain was made to fail once
    c.close()
