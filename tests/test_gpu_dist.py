"""Row-block distributed algebra on the GPU (include/ab2_dist.h) against the oracle.

R ranks run on cuda:0 as a local group: one host thread and one context per
rank (ctypes releases the GIL, so the threads run concurrently), meeting at
host barriers; no kernel waits for another rank.  Everything is bit for bit:
the layout and exchange plan (DistStructInfo), the SpMV with its halo
(local sum, then + ghost sum), the rank-ordered dots (each rank's libab2 tree
over its rows), block-Jacobi ILU(0) (the reference's parallel factorisation),
the device-resident distributed CG, and the reference's OWN CG/BiCGStab
templates running on Alien::B200::DistAlgebra in R threads
(tests/cpp/dist_drop_in).  Failure detection: a rank that never reaches a
collective makes the others fail with AB2_ERR_TIMEOUT at the host barrier.
"""
import json
import subprocess
import threading
from pathlib import Path

import numpy as np
import pytest

from alien_b200 import abi
from oracle import oracle as O
from tests import problems

pytestmark = pytest.mark.gpu

BIN = Path(__file__).resolve().parent / "cpp" / "_build" / "dist_drop_in"


def run_ranks(k, fn, timeout_s=60.0):
    """fn(rank, ctx, comm) on k threads over a local group; returns the results in rank order."""
    ctxs = [abi.Context(0) for _ in range(k)]
    comms = abi.Comm.local_group(ctxs, timeout_s=timeout_s)
    out, err = [None] * k, [None] * k

    def body(r):
        try:
            out[r] = fn(r, ctxs[r], comms[r])
        except BaseException as e:  # noqa: BLE001 - reported below
            err[r] = e

    ts = [threading.Thread(target=body, args=(r,)) for r in range(k)]
    for t in ts:
        t.start()
    for t in ts:
        t.join()
    for c in comms:
        c.close()
    for e in err:
        if e is not None:
            raise e
    return out


def tree_blocks():
    return abi.Context(0).info.reduction_max_blocks


CASES = [("diffusion12", 2, 144), ("diffusion12", 3, 144), ("poisson16", 4, 1), ("ragged", 3, 1),
         ("convdiff_10x11x12", 2, 110)]


@pytest.mark.parametrize("name,k,align", CASES)
def test_layout_and_plan_match_oracle(name, k, align):
    P = problems.get(name)
    off = abi.row_offsets(P.n, k, align)

    def rank(r, ctx, comm):
        A = abi.DistMatrix.from_global(ctx, comm, off, P.row_ptr, P.cols, P.vals)
        return A.layout(), A.plan(), A.info

    res = run_ranks(k, rank)
    for r, (lay, plan, info) in enumerate(res):
        ref = O.dist_layout(P.row_ptr, P.cols, P.vals, off, r)
        for key in ref:
            np.testing.assert_array_equal(lay[key], ref[key], err_msg=f"rank {r} {key}")
        # the plan: ghost slices per owner, and every send list is what the receiver asked for
        owners = np.searchsorted(off, ref["ghost_uids"], side="right") - 1
        assert list(plan["recv_ranks"]) == sorted(set(owners.tolist()))
        for q, (a, b) in zip(plan["recv_ranks"], zip(plan["recv_offsets"][:-1], plan["recv_offsets"][1:])):
            theirs = res[q][1]
            j = list(theirs["send_ranks"]).index(r)
            ids = theirs["send_ids"][theirs["send_offsets"][j]:theirs["send_offsets"][j + 1]] + off[q]
            np.testing.assert_array_equal(ids, ref["ghost_uids"][a:b])
        assert info.local_rows == off[r + 1] - off[r] and info.ghost_rows == ref["ghost_uids"].size


@pytest.mark.parametrize("name,k,align", CASES + [("poisson16", 1, 1)])
def test_dist_mult_dot_norms_bit_exact(name, k, align):
    P = problems.get(name)
    off = abi.row_offsets(P.n, k, align)
    rng = np.random.default_rng(7)
    x, y = rng.uniform(-1, 1, P.n), rng.standard_normal(P.n)
    tb = tree_blocks()

    def rank(r, ctx, comm):
        A = abi.DistMatrix.from_global(ctx, comm, off, P.row_ptr, P.cols, P.vals)
        a, b = off[r], off[r + 1]
        xv, yv, zv = A.vector(x[a:b]), A.vector(y[a:b]), A.vector()
        outs = []
        for _ in range(3):  # repeated exchanges reuse both parities of the buffers
            A.mult(xv, zv)
            outs.append(zv.download())
        return outs, comm.dot(xv, yv), comm.norm2(xv), comm.norm1(yv)

    res = run_ranks(k, rank)
    exp = O.dist_spmv(P.row_ptr, P.cols, P.vals, off, x)
    for t in range(3):
        np.testing.assert_array_equal(np.concatenate([o[0][t] for o in res]), exp)
    d = O.dist_dot(off, x, y, O.DOT_DEVICE_TREE, tb)
    n2 = np.sqrt(O.dist_dot(off, x, x, O.DOT_DEVICE_TREE, tb))
    for o in res:  # identical on every rank
        assert o[1] == d and o[2] == n2
        assert o[3] == pytest.approx(np.abs(y).sum(), rel=1e-12)


@pytest.mark.parametrize("name,k,align,schedule", [("diffusion12", 2, 144, "stencil"), ("diffusion12", 3, 144, "auto"),
                                                   ("diffusion12", 3, 144, "wavefront"), ("ragged", 3, 1, "auto"),
                                                   ("convdiff_10x11x12", 4, 1, "auto"), ("poisson16", 1, 1, "auto")])
def test_block_ilu0_bit_exact(name, k, align, schedule):
    P = problems.get(name)
    off = abi.row_offsets(P.n, k, align)
    y = np.random.default_rng(9).standard_normal(P.n)

    def rank(r, ctx, comm):
        A = abi.DistMatrix.from_global(ctx, comm, off, P.row_ptr, P.cols, P.vals)
        M = abi.DistPrecond(ctx, A, "ilu0", ilu_schedule=schedule)
        yv, xv = A.vector(y[off[r]:off[r + 1]]), A.vector()
        outs = []
        for _ in range(2):  # the sweeps leave their state ready for the next application
            M.apply(yv, xv)
            outs.append(xv.download())
        return outs, M.ilu0_values(), M.info.ilu_schedule

    res = run_ranks(k, rank)
    x, parts = O.bj_ilu0_apply(P.row_ptr, P.cols, P.vals, off, y)
    for t in range(2):
        np.testing.assert_array_equal(np.concatenate([o[0][t] for o in res]), x)
    for r, o in enumerate(res):
        np.testing.assert_array_equal(o[1], parts[r])
        if schedule == "stencil":
            assert o[2] == 2


SOLVER_CASES = [("diffusion12", 1, 144, "ilu0"), ("diffusion12", 2, 144, "ilu0"),
                                                  ("diffusion12", 3, 144, "diag"), ("poisson16", 4, 1, "ilu0"),
                                                  ("ragged", 3, 1, "ilu0"), ("poisson16", 2, 1, "none"),
                                                  # eight ranks sharing the GPU: the transfer streams of a local
                                                  # group lag their contexts, which once let a gather overwrite
                                                  # partials before the previous sum had read them
                ("diffusion64", 8, 4096, "ilu0"), ("diffusion64", 8, 4096, "diag")]


@pytest.mark.parametrize("solver,name,k,align,precond",
                         [("cg",) + c for c in SOLVER_CASES] +
                         [("bicgs", "convdiff_10x11x12", 1, 110, "ilu0"), ("bicgs", "convdiff_10x11x12", 3, 110, "ilu0"),
                          ("bicgs", "ragged", 2, 1, "diag"), ("bicgs", "convdiff16", 4, 256, "ilu0"),
                          ("bicgs", "diffusion64", 8, 4096, "ilu0"), ("bicgs", "poisson16", 2, 1, "none")])
def test_dist_solver_bit_exact(solver, name, k, align, precond):
    P = problems.get(name)
    off = abi.row_offsets(P.n, k, align)
    tb = tree_blocks()

    def rank(r, ctx, comm):
        A = abi.DistMatrix.from_global(ctx, comm, off, P.row_ptr, P.cols, P.vals)
        S = abi.DistSolver(ctx, comm, A, solver=solver, precond=precond, tol=1e-8, max_iter=400)
        b, x = A.vector(P.b[off[r]:off[r + 1]]), A.vector()
        st = S.solve(b, x)
        return st, x.download(), S.history()

    res = run_ranks(k, rank)
    o = O.dist_solve(P.row_ptr, P.cols, P.vals, off, P.b, solver=solver, precond=precond, tol=1e-8, max_iter=400,
                     dot_mode=O.DOT_DEVICE_TREE, tree_blocks=tb)
    for st, _, h in res:
        assert (st.iterations, st.succeeded, st.breakdown) == (o.iterations, o.converged, o.breakdown)
        np.testing.assert_array_equal(h, o.history)
    np.testing.assert_array_equal(np.concatenate([r[1] for r in res]), o.x)
    if o.converged and solver == "cg":
        assert res[0][0].true_residual < 1e-7


@pytest.mark.skipif(not BIN.exists(), reason="tests/cpp/_build/dist_drop_in not built (reference sources absent)")
@pytest.mark.parametrize("name,k,align,solver,pc", [("diffusion12", 2, 144, "cg", "ilu0"), ("diffusion12", 3, 144, "cg", "diag"),
                                                     ("convdiff_10x11x12", 3, 110, "bicgs", "ilu0"),
                                                     ("ragged", 2, 1, "bicgs", "diag"), ("poisson16", 4, 1, "cg", "ilu0"),
                                                     ("diffusion24", 8, 576, "bicgs", "ilu0")])
def test_reference_templates_on_dist_algebra(tmp_path, name, k, align, solver, pc):
    P = problems.get(name)
    off = abi.row_offsets(P.n, k, align)
    P.row_ptr.astype(np.int32).tofile(tmp_path / "rp.i32")
    P.cols.astype(np.int32).tofile(tmp_path / "ci.i32")
    P.vals.astype(np.float64).tofile(tmp_path / "v.f64")
    P.b.astype(np.float64).tofile(tmp_path / "b.f64")
    off.astype(np.int32).tofile(tmp_path / "off.i32")
    out = subprocess.run([str(BIN), str(tmp_path), solver, pc, "1e-8", "400"], capture_output=True, text=True,
                         timeout=300)
    assert out.returncode == 0, out.stderr
    res = json.loads(out.stdout.strip().splitlines()[-1])
    o = O.dist_solve(P.row_ptr, P.cols, P.vals, off, P.b, solver=solver, precond=pc, tol=1e-8, max_iter=400,
                     dot_mode=O.DOT_DEVICE_TREE, tree_blocks=tree_blocks())
    assert (res["iterations"], res["converged"], res["ranks"]) == (o.iterations, o.converged, k)
    np.testing.assert_array_equal(np.fromfile(tmp_path / "x.f64", dtype=np.float64), o.x)
    assert res["gpu_launches"] > 2 * res["iterations"]


def test_nccl_single_rank_matches_local_group():
    try:
        uid = abi.Comm.nccl_unique_id()
    except abi.AB2Error as e:
        pytest.skip(f"NCCL not loadable: {e}")
    P = problems.get("diffusion12")
    off = np.asarray([0, P.n], np.int32)
    ctx = abi.Context(0)
    comm = abi.Comm.nccl(ctx, uid, 0, 1)
    A = abi.DistMatrix.from_global(ctx, comm, off, P.row_ptr, P.cols, P.vals)
    S = abi.DistSolver(ctx, comm, A, solver="cg", precond="ilu0", tol=1e-8, max_iter=400)
    b, x = A.vector(P.b), A.vector()
    st = S.solve(b, x)
    got = x.download()
    S.close()
    A.close()
    comm.close()
    (st2, x2, _), = run_ranks(1, lambda r, c, m: _solve_one(c, m, off, P))
    assert st.iterations == st2.iterations
    np.testing.assert_array_equal(got, x2)


def _solve_one(ctx, comm, off, P):
    A = abi.DistMatrix.from_global(ctx, comm, off, P.row_ptr, P.cols, P.vals)
    S = abi.DistSolver(ctx, comm, A, solver="cg", precond="ilu0", tol=1e-8, max_iter=400)
    b, x = A.vector(P.b), A.vector()
    return S.solve(b, x), x.download(), None


def test_rank_that_never_arrives_times_out_on_the_host():
    """Failure detection without a GPU fault: rank 1 leaves between steps;
    rank 0's next collective gives up at the host barrier (AB2_ERR_TIMEOUT)
    and every later collective fails at once."""
    P = problems.get("poisson16")
    off = abi.row_offsets(P.n, 2)

    def rank(r, ctx, comm):
        A = abi.DistMatrix.from_global(ctx, comm, off, P.row_ptr, P.cols, P.vals)
        x = A.vector(np.ones(off[r + 1] - off[r]))
        comm.dot(x, x)  # one step together
        if r == 1:
            return "left"
        codes = []
        for _ in range(2):
            try:
                comm.dot(x, x)
            except abi.AB2Error as e:
                codes.append(e.code)
        ctx.synchronize()  # the context stays usable
        return codes

    res = run_ranks(2, rank, timeout_s=1.0)
    assert res[1] == "left"
    assert res[0] == [abi.AB2_ERR_TIMEOUT, abi.AB2_ERR_TIMEOUT]


@pytest.mark.parametrize("solver", ["cg", "bicgs"])
def test_dist_breakdown_reported(solver):
    """The zero operator on two ranks: p.Ap (CG) or v.r0 (BiCGStab) sums to 0
    on every rank alike, the stop test fails, breakdown "alpha" (CG.h:96-104,
    BiCGStab.h:186-187), the same on every rank and in the oracle."""
    n = 64
    rp = np.arange(n + 1, dtype=np.int32)
    ci = np.arange(n, dtype=np.int32)
    vals = np.zeros(n)
    off = abi.row_offsets(n, 2)

    def rank(r, ctx, comm):
        A = abi.DistMatrix.from_global(ctx, comm, off, rp, ci, vals)
        S = abi.DistSolver(ctx, comm, A, solver=solver, precond="none", tol=1e-8, max_iter=10)
        st = S.solve(A.vector(np.ones(off[r + 1] - off[r])), A.vector())
        return st

    res = run_ranks(2, rank)
    o = O.dist_solve(rp, ci, vals, off, np.ones(n), solver=solver, precond="none", tol=1e-8, max_iter=10)
    assert o.error == -3 and o.breakdown == "alpha"
    for st in res:
        assert st.error == abi.AB2_ERR_BREAKDOWN and st.breakdown == "alpha"
        assert st.iterations == o.iterations and not st.succeeded


def test_rows_rejected_on_one_rank_fail_every_rank():
    """A rank whose rows are invalid still takes part in the set-up exchange,
    so every rank fails with AB2_ERR_BAD_ARG at once (no rank left waiting)."""
    P = problems.get("poisson16")
    off = abi.row_offsets(P.n, 2)

    def rank(r, ctx, comm):
        a, b = int(off[r]), int(off[r + 1])
        lo, hi = int(P.row_ptr[a]), int(P.row_ptr[b])
        cols = P.cols[lo:hi].copy()
        if r == 1:
            cols[3] = P.n + 5  # out of range
        try:
            abi.DistMatrix(ctx, comm, off, P.row_ptr[a:b + 1] - lo, cols, P.vals[lo:hi])
        except abi.AB2Error as e:
            return e.code
        return None

    assert run_ranks(2, rank, timeout_s=30.0) == [abi.AB2_ERR_BAD_ARG, abi.AB2_ERR_BAD_ARG]
