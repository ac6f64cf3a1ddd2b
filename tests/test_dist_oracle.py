"""The row-block distributed algebra's oracle, on CPU (no GPU).

* the layout (DistStructInfo + sortGhostCols) against a second, independent
  restatement written here with Python sets and dicts;
* the SpMV (_parallelMult: local sum, then + ghost sum) against plain Python
  floats, and the rank-ordered dot;
* block-Jacobi ILU(0) against the reference's OWN parallel
  LUFactorisationAlgo branch (ILU0Preconditioner.h:93-119, 181-231), compiled
  from its header into oracle/_ref: bit for bit, factor and application;
* one rank = the sequential solve, bit for bit;
* two real processes (gloo) exchanging ghost values and partial dots with
  torch.distributed reproduce the oracle's distributed CG bit for bit: the
  host-side protocol the GPU ranks follow (requests, send lists, halo, rank-
  ordered sums).
"""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from alien_b200 import abi
from oracle import oracle as O
from tests import problems

CASES = [("poisson16", [0, 1000, 2048, 4096]), ("ragged", None), ("diffusion12", [0, 576, 1728]),
         ("convdiff_10x11x12", [0, 110, 700, 1000, 1320])]


def offsets_for(P, off):
    return np.asarray(off if off is not None else abi.row_offsets(P.n, 3), dtype=np.int32)


def py_layout(P, off, r):
    """DistStructInfo::compute restated with sets (independent of the oracle's C++)."""
    base, end = int(off[r]), int(off[r + 1])
    owner = lambda c: int(np.searchsorted(off, c, side="right") - 1)
    gids = {}
    rows = []
    for g in range(base, end):
        cs = P.cols[P.row_ptr[g]:P.row_ptr[g + 1]]
        vs = P.vals[P.row_ptr[g]:P.row_ptr[g + 1]]
        loc = [(int(c) - base, float(v)) for c, v in zip(cs, vs) if base <= c < end]
        gh = [(int(c), float(v)) for c, v in zip(cs, vs) if not base <= c < end]
        for c, _ in gh:
            gids.setdefault(owner(c), set()).add(c)
        rows.append((loc, gh))
    uids = [u for q in sorted(gids) for u in sorted(gids[q])]
    gid_of = {u: (end - base) + i for i, u in enumerate(uids)}
    rp, ci, vv, lrs, iface = [0], [], [], [], []
    for i, (loc, gh) in enumerate(rows):
        ci += [c for c, _ in loc] + [gid_of[c] for c, _ in gh]
        vv += [v for _, v in loc] + [v for _, v in gh]
        lrs.append(len(loc))
        rp.append(len(ci))
        if gh:
            iface.append(i)
    return dict(row_ptr=rp, cols=ci, vals=vv, local_row_size=lrs, ghost_uids=uids, interface_rows=iface)


@pytest.mark.parametrize("name,off", CASES)
def test_layout_matches_independent_restatement(name, off):
    P = problems.get(name)
    off = offsets_for(P, off)
    for r in range(off.size - 1):
        a = O.dist_layout(P.row_ptr, P.cols, P.vals, off, r)
        b = py_layout(P, off, r)
        for k in b:
            np.testing.assert_array_equal(a[k], np.asarray(b[k], dtype=a[k].dtype), err_msg=f"{name} rank {r} {k}")


@pytest.mark.parametrize("name,off", CASES)
def test_dist_spmv_is_local_sum_then_ghost_sum(name, off):
    P = problems.get(name)
    off = offsets_for(P, off)
    x = np.random.default_rng(3).uniform(-1, 1, P.n)
    y = O.dist_spmv(P.row_ptr, P.cols, P.vals, off, x)
    exp = np.empty(P.n)
    for r in range(off.size - 1):
        base, end = int(off[r]), int(off[r + 1])
        for g in range(base, end):
            cs = P.cols[P.row_ptr[g]:P.row_ptr[g + 1]]
            vs = P.vals[P.row_ptr[g]:P.row_ptr[g + 1]]
            t = 0.0
            for c, v in zip(cs, vs):
                if base <= c < end:
                    t += float(v) * float(x[c])
            u, any_ghost = 0.0, False
            for c, v in zip(cs, vs):
                if not base <= c < end:
                    u += float(v) * float(x[c])
                    any_ghost = True
            exp[g] = t + u if any_ghost else t
    np.testing.assert_array_equal(y, exp)
    # one rank: the sequential SpMV
    np.testing.assert_array_equal(O.dist_spmv(P.row_ptr, P.cols, P.vals, [0, P.n], x),
                                  O.spmv(P.row_ptr, P.cols, P.vals, x))


def test_dist_dot_is_rank_ordered_sum_of_local_dots():
    rng = np.random.default_rng(5)
    x, y = rng.standard_normal(10007), rng.standard_normal(10007)
    off = abi.row_offsets(x.size, 4)
    for mode, tb in ((O.DOT_SEQUENTIAL, 1184), (O.DOT_DEVICE_TREE, 1184), (O.DOT_DEVICE_TREE, 7)):
        parts = [O.dot(x[a:b], y[a:b]) if mode == O.DOT_SEQUENTIAL else O.dot_tree(x[a:b], y[a:b], tb)
                 for a, b in zip(off[:-1], off[1:])]
        s = parts[0]
        for p in parts[1:]:
            s = s + p
        assert O.dist_dot(off, x, y, mode, tb) == s


@pytest.mark.skipif(not O.ref_available(), reason="oracle/_ref not built")
@pytest.mark.parametrize("name,off", CASES)
def test_block_ilu0_matches_reference_parallel_branch(name, off):
    P = problems.get(name)
    off = offsets_for(P, off)
    y = np.random.default_rng(11).standard_normal(P.n)
    x, parts = O.bj_ilu0_apply(P.row_ptr, P.cols, P.vals, off, y)
    for r in range(off.size - 1):
        L = O.dist_layout(P.row_ptr, P.cols, P.vals, off, r)
        xr, lur = O.ref_bj_ilu0_apply(L, y[off[r]:off[r + 1]])
        np.testing.assert_array_equal(xr, x[off[r]:off[r + 1]])
        loc = np.concatenate([lur[s:s + m] for s, m in zip(L["row_ptr"][:-1], L["local_row_size"])])
        np.testing.assert_array_equal(loc, parts[r])


def test_block_ilu0_bound_of_the_reference_is_reproduced():
    """ILU0Preconditioner.h:107 bounds row i's elimination by kcol[krow] +
    local_row_size[i]: on a 7-point matrix that leaves only the divisions
    (U keeps A's upper part, the diagonal is untouched); where a short row
    precedes a long one some updates survive."""
    P = problems.get("poisson16")
    off = [0, 2048, 4096]
    _, parts = O.bj_ilu0_apply(P.row_ptr, P.cols, P.vals, off, np.ones(P.n))
    for r in range(2):
        L = O.dist_layout(P.row_ptr, P.cols, P.vals, off, r)
        vloc = np.concatenate([L["vals"][s:s + m] for s, m in zip(L["row_ptr"][:-1], L["local_row_size"])])
        lu = parts[r]
        rows = np.repeat(np.arange(L["local_row_size"].size), L["local_row_size"])
        cloc = np.concatenate([L["cols"][s:s + m] for s, m in zip(L["row_ptr"][:-1], L["local_row_size"])])
        upper = cloc >= rows
        np.testing.assert_array_equal(lu[upper], vloc[upper])  # diagonal and U untouched
        assert not np.array_equal(lu, vloc)                      # L divided by the pivots
    # short rows followed by long ones: there the bound lets updates through
    R = short_long_matrix()
    off = [0, 10, 20]
    _, parts = O.bj_ilu0_apply(R.row_ptr, R.cols, R.vals, off, np.ones(R.n))
    changed_upper = 0
    for r in range(2):
        L = O.dist_layout(R.row_ptr, R.cols, R.vals, off, r)
        vloc = np.concatenate([L["vals"][s:s + m] for s, m in zip(L["row_ptr"][:-1], L["local_row_size"])])
        rows = np.repeat(np.arange(L["local_row_size"].size), L["local_row_size"])
        cloc = np.concatenate([L["cols"][s:s + m] for s, m in zip(L["row_ptr"][:-1], L["local_row_size"])])
        changed_upper += int(np.sum(parts[r][cloc >= rows] != vloc[cloc >= rows]))
    assert changed_upper > 0


def short_long_matrix(n: int = 20) -> abi.CsrProblem:
    """Even rows: diagonal and the next column; odd rows: the previous column,
    the diagonal and up to three more on the right (diagonally dominant)."""
    rp, ci, vv = [0], [], []
    for i in range(n):
        cols = [i, i + 1] if i % 2 == 0 else [i - 1, i, i + 1, i + 2, i + 3]
        cols = [c for c in cols if c < n]
        for c in cols:
            ci.append(c)
            vv.append(8.0 + 0.1 * i if c == i else -1.0 - 0.01 * (i + 2 * c))
        rp.append(len(ci))
    rp, ci, vv = np.asarray(rp, np.int32), np.asarray(ci, np.int32), np.asarray(vv)
    return abi.CsrProblem(n=n, row_ptr=rp, cols=ci, vals=vv, x_true=None, b=np.ones(n), log10_k=None, shape=(n, 1, 1))


@pytest.mark.skipif(not O.ref_available(), reason="oracle/_ref not built")
def test_block_ilu0_with_surviving_updates_matches_reference():
    R = short_long_matrix()
    for off in ([0, 10, 20], [0, 7, 13, 20]):
        y = np.linspace(-1, 2, R.n)
        x, parts = O.bj_ilu0_apply(R.row_ptr, R.cols, R.vals, off, y)
        for r in range(len(off) - 1):
            L = O.dist_layout(R.row_ptr, R.cols, R.vals, off, r)
            xr, lur = O.ref_bj_ilu0_apply(L, y[off[r]:off[r + 1]])
            np.testing.assert_array_equal(xr, x[off[r]:off[r + 1]])
            loc = np.concatenate([lur[s:s + m] for s, m in zip(L["row_ptr"][:-1], L["local_row_size"])])
            np.testing.assert_array_equal(loc, parts[r])


@pytest.mark.parametrize("solver,precond", [("cg", "diag"), ("cg", "ilu0"), ("bicgs", "ilu0"), ("cg", "none")])
def test_one_rank_is_the_sequential_solve(solver, precond):
    P = problems.get("diffusion12")
    a = O.dist_solve(P.row_ptr, P.cols, P.vals, [0, P.n], P.b, solver=solver, precond=precond, max_iter=300)
    b = O.solve(P.row_ptr, P.cols, P.vals, P.b, solver=solver, precond=precond, max_iter=300)
    assert (a.iterations, a.converged) == (b.iterations, b.converged)
    np.testing.assert_array_equal(a.history, b.history)
    np.testing.assert_array_equal(a.x, b.x)


@pytest.mark.parametrize("name,precond", [("diffusion12", "ilu0"), ("poisson16", "ilu0"), ("diffusion12", "diag")])
def test_block_jacobi_solves_converge_to_the_same_solution(name, precond):
    P = problems.get(name)
    ref = O.solve(P.row_ptr, P.cols, P.vals, P.b, precond=precond, tol=1e-12, max_iter=2000)
    its = []
    for k in (2, 3, 4):
        r = O.dist_solve(P.row_ptr, P.cols, P.vals, abi.row_offsets(P.n, k), P.b, precond=precond, tol=1e-10)
        assert r.converged
        its.append(r.iterations)
        res = P.b - O.spmv(P.row_ptr, P.cols, P.vals, r.x)
        assert np.linalg.norm(res) <= 1e-9 * np.linalg.norm(P.b)
        assert np.linalg.norm(r.x - ref.x) <= 1e-5 * np.linalg.norm(ref.x)
    if precond == "ilu0":  # block Jacobi weakens ILU(0) as the blocks shrink
        assert its[-1] >= its[0]


# ---------------------------------------------------------------- two gloo processes
def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _gloo_rank(rank: int, world: int, port: int, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    import datetime

    import torch
    import torch.distributed as dist

    try:
        dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=60))
        P = problems.get("diffusion12")
        off = abi.row_offsets(P.n, world, align=144)
        base, end = int(off[rank]), int(off[rank + 1])
        n = end - base
        L = O.dist_layout(P.row_ptr, P.cols, P.vals, off, rank)
        # requests: which of my ghosts each owner holds (ascending), exchanged like DistStructInfo
        uids = L["ghost_uids"]
        owner = np.searchsorted(off, uids, side="right") - 1
        req = {int(q): uids[owner == q].tolist() for q in np.unique(owner)}
        allreq = [None] * world
        dist.all_gather_object(allreq, req)
        send = {q: np.asarray(allreq[q][rank]) - base for q in range(world) if q != rank and rank in allreq[q]}
        recv = {q: (int(np.searchsorted(uids, req[q][0])), len(req[q])) for q in req}
        # diagonal block CSR (local entries) and ghost entries
        rp, ci, vv, lrs = L["row_ptr"], L["cols"], L["vals"], L["local_row_size"]
        lrp = np.concatenate([[0], np.cumsum(lrs)]).astype(np.int32)
        lci = np.concatenate([ci[s:s + m] for s, m in zip(rp[:-1], lrs)]).astype(np.int32)
        lv = np.concatenate([vv[s:s + m] for s, m in zip(rp[:-1], lrs)])
        inv = np.array([1.0 / lv[lrp[i] + int(np.searchsorted(lci[lrp[i]:lrp[i + 1]], i))] for i in range(n)])

        def halo(x):
            ghosts = np.empty(uids.size)
            ops = []
            for q, ids in send.items():
                ops.append(dist.isend(torch.from_numpy(np.ascontiguousarray(x[ids])), q))
            bufs = {}
            for q, (s, m) in recv.items():
                bufs[q] = torch.empty(m, dtype=torch.float64)
                ops.append(dist.irecv(bufs[q], q))
            for op in ops:
                op.wait()
            for q, (s, m) in recv.items():
                ghosts[s:s + m] = bufs[q].numpy()
            return ghosts

        def mult(x):
            g = halo(x)
            y = O.spmv(lrp, lci, lv, x)
            for i in L["interface_rows"]:
                t = 0.0
                for k in range(rp[i] + lrs[i], rp[i + 1]):
                    t += float(vv[k]) * float(g[ci[k] - n])
                y[i] = y[i] + t
            return y

        def gdot(x, y):
            parts = [None] * world
            dist.all_gather_object(parts, O.dot(x, y))
            s = parts[0]
            for p in parts[1:]:
                s = s + p
            return s

        # CG.h with Diag (the oracle's restatement of the template, run by two processes)
        b = P.b[base:end].copy()
        x = np.zeros(n)
        tol, max_iter = 1e-8, 300
        criteria = tol * tol * gdot(b, b)
        r = b.copy()
        r = O.axpy(-1.0, mult(x), r)
        z = inv * r
        rho1 = gdot(r, z)
        p = z.copy()
        q = mult(p)
        alpha = rho1 / gdot(p, q)
        x = O.axpy(alpha, p, x)
        r = O.axpy(-alpha, q, r)
        rho, it, hist = rho1, 1, []
        while True:
            rr = gdot(r, r)
            hist.append(rr)
            if rr < criteria or it >= max_iter:
                break
            z = inv * r
            rho1 = gdot(r, z)
            z = O.axpy(rho1 / rho, p, z)
            p = z.copy()
            q = mult(p)
            alpha = rho1 / gdot(q, p)
            x = O.axpy(alpha, p, x)
            r = O.axpy(-alpha, q, r)
            rho = rho1
            it += 1
        out.put((rank, it, x, np.asarray(hist)))
        dist.destroy_process_group()
    except Exception as e:  # reported to the parent
        out.put((rank, "error", repr(e), None))


def test_two_gloo_ranks_reproduce_the_distributed_cg():
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_gloo_rank, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = {}
    for _ in range(world):
        rank, it, x, h = q.get(timeout=240)
        assert it != "error", x
        res[rank] = (it, x, h)
    for p in procs:
        p.join(timeout=60)
    P = problems.get("diffusion12")
    off = abi.row_offsets(P.n, world, align=144)
    o = O.dist_solve(P.row_ptr, P.cols, P.vals, off, P.b, solver="cg", precond="diag", tol=1e-8, max_iter=300)
    assert res[0][0] == res[1][0] == o.iterations
    np.testing.assert_array_equal(np.concatenate([res[0][1], res[1][1]]), o.x)
    np.testing.assert_array_equal(res[0][2], o.history)
