"""Batched uneven systems in one persistent launch, vs the oracle.

No counterpart in the reference; parity is against this repo's restatement
(oracle/ab2_oracle.cpp orc_batch_solve: per system, CG.h's Jacobi-PCG in FP32
inside FP64 refinement, every dot reduced as one thread-block cluster of the
given size and width reduces it).  For each fixed configuration the GPU must
reproduce it bit for bit: per-system convergence flags, refinement steps, FP32
iteration counts, residuals and every solution value.
"""
import numpy as np
import pytest

from alien_b200 import abi
from oracle import oracle as O

pytestmark = pytest.mark.gpu

F32 = abi.FMT_CSR | abi.FMT_ELL | abi.FMT_F32


@pytest.fixture(scope="module")
def batch():
    return abi.batch_problem(nsys=24, min_rows=300, max_rows=6000, seed=3)


def run(ctx, B, **kw):
    P = B.problem
    A = ctx.matrix(P.row_ptr, P.cols, P.vals, F32)
    S = abi.Batch(ctx, A, B.sys_offsets, **kw)
    b, x = ctx.vector(P.b), ctx.vector(P.n)
    st = S.solve(b, x)
    return S, st, x.download()


@pytest.mark.parametrize("variant,cluster,threads,shape", [(abi.SPMV_ELL, 4, 256, 32), (abi.SPMV_ELL, 1, 128, 32),
                                                           (abi.SPMV_ELL, 8, 512, 32), (abi.SPMV_ELL, 4, 256, 16),
                                                           (abi.SPMV_ELL, 2, 512, 64),
                                                           (abi.SPMV_CSR_SCALAR, 2, 256, 1),
                                                           (abi.SPMV_CSR_SCALAR, 8, 1024, 1),
                                                           (abi.SPMV_CSR_SCALAR, 4, 256, 2),
                                                           (abi.SPMV_CSR_SCALAR, 2, 512, 4),
                                                           (abi.SPMV_CSR_SCALAR, 8, 256, 8)])
def test_batch_bit_exact(ctx, batch, variant, cluster, threads, shape):
    """shape: rows per ELL slice, or CSR lanes per row (the latter sums a row
    in a lane tree: the oracle restates it)."""
    ell = variant == abi.SPMV_ELL
    S, st, x = run(ctx, batch, tol=1e-8, spmv_variant=variant, cluster_size=cluster, threads=threads,
                   ell_slice=shape if ell else 0, lanes_per_row=0 if ell else shape)
    info = S.info
    assert not info.tuned and (info.cluster_size, info.threads) == (cluster, threads)
    assert (info.ell_slice, info.lanes_per_row) == ((shape, 0) if ell else (0, shape))
    P = batch.problem
    o = O.batch_solve(P.row_ptr, P.cols, P.vals, batch.sys_offsets, P.b, tol=1e-8, cluster_size=cluster,
                      threads=threads, lanes_per_row=1 if ell else shape)
    conv, outer, inner, res = S.results()
    np.testing.assert_array_equal(conv, o.converged)
    np.testing.assert_array_equal(outer, o.outer)
    np.testing.assert_array_equal(inner, o.inner)
    np.testing.assert_array_equal(res, o.residual)
    np.testing.assert_array_equal(x, o.x)
    assert st.systems_converged == batch.nsys and st.max_residual < 1e-8
    assert st.inner_total == int(inner.sum())


def test_batch_autotuner_picks_the_fastest_trial(ctx, batch):
    """Round 1: the seven inner SpMV formats (ELL with 16 / 32 / 64 rows per
    slice, CSR with 1 / 2 / 4 / 8 lanes per row) at 8 CTAs x 512 threads;
    round 2: the best of them at every placeable cluster size (1, 2, 4, 8
    always, 16 where the GPU places it) x width (256, 512)."""
    S, st, x = run(ctx, batch, tol=1e-8)
    info = S.info
    trials = S.trials()
    assert info.tuned and len(trials) == info.trials and 7 + 4 * 2 - 1 <= len(trials) <= 7 + 5 * 2 - 1
    fmts = {(t[0], t[4], t[5]) for t in trials[:7]}
    assert fmts == {(abi.SPMV_ELL, 16, 0), (abi.SPMV_ELL, 32, 0), (abi.SPMV_ELL, 64, 0),
                    (abi.SPMV_CSR_SCALAR, 0, 1), (abi.SPMV_CSR_SCALAR, 0, 2), (abi.SPMV_CSR_SCALAR, 0, 4),
                    (abi.SPMV_CSR_SCALAR, 0, 8)}
    best = min(trials, key=lambda t: t[3])
    assert (info.spmv_variant, info.cluster_size, info.threads) == best[:3]
    assert (info.ell_slice, info.lanes_per_row) == best[4:]
    P = batch.problem
    o = O.batch_solve(P.row_ptr, P.cols, P.vals, batch.sys_offsets, P.b, tol=1e-8, cluster_size=info.cluster_size,
                      threads=info.threads, lanes_per_row=info.lanes_per_row if info.lanes_per_row else 1)
    np.testing.assert_array_equal(x, o.x)
    assert st.systems_converged == batch.nsys


def test_batch_per_system_convergence_and_error(ctx, batch):
    """Every system reaches its own tolerance; a system with a zero right-hand
    side is done at once; each solution is close to a plain FP64 solve."""
    P = batch.problem
    b = P.b.copy()
    z0, z1 = batch.sys_offsets[5], batch.sys_offsets[6]
    b[z0:z1] = 0.0
    A = ctx.matrix(P.row_ptr, P.cols, P.vals, F32)
    S = abi.Batch(ctx, A, batch.sys_offsets, tol=1e-9, cluster_size=2, threads=256, spmv_variant=abi.SPMV_ELL)
    vb, vx = ctx.vector(b), ctx.vector(P.n)
    st = S.solve(vb, vx)
    x = vx.download()
    conv, outer, inner, res = S.results()
    assert conv.all() and outer[5] == 0 and inner[5] == 0 and np.all(x[z0:z1] == 0)
    assert np.all(res[np.arange(batch.nsys) != 5] < 1e-9)
    for s in (0, 7, 13):
        a, e = batch.sys_offsets[s], batch.sys_offsets[s + 1]
        rp = P.row_ptr[a:e + 1] - P.row_ptr[a]
        ci = P.cols[P.row_ptr[a]:P.row_ptr[e]] - a
        vv = P.vals[P.row_ptr[a]:P.row_ptr[e]]
        x64 = O.solve(rp, ci, vv, b[a:e], solver="cg", precond="ilu0", tol=1e-13, max_iter=3000).x
        assert np.linalg.norm(x[a:e] - x64) / np.linalg.norm(x64) < 1e-6


def test_batch_rejects_bad_input(ctx, batch):
    P = batch.problem
    A32 = ctx.matrix(P.row_ptr, P.cols, P.vals, F32)
    A64 = ctx.matrix(P.row_ptr, P.cols, P.vals)
    for args, kw in [((A64, batch.sys_offsets), {}),  # no FP32 values
                     ((A32, np.array([0, P.n // 2, P.n // 2, P.n])), {}),  # empty system
                     ((A32, np.array([0, batch.sys_offsets[1] + 1, P.n])), {}),  # cuts through a block
                     ((A32, batch.sys_offsets), dict(cluster_size=3)),
                     ((A32, batch.sys_offsets), dict(threads=100)),
                     ((A32, batch.sys_offsets), dict(ell_slice=8)),
                     ((A32, batch.sys_offsets), dict(lanes_per_row=3))]:
        with pytest.raises(abi.AB2Error) as e:
            abi.Batch(ctx, *args, **kw)
        assert e.value.code == abi.AB2_ERR_BAD_ARG
