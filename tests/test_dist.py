"""Multi-rank plumbing on CPU: two gloo ranks, as bench.py runs N GPUs.

Each rank builds its own seeded system (seed = rank: weak scaling, no
collective on the data path), solves it with the CPU oracle, and the ranks
combine their timings exactly as the bench does (barrier, max over ranks) and
their work (sum).  Also checks that a rank that raises leaves the others with
an error rather than a hang (short process-group timeout).
"""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank: int, world: int, port: int, out, mode: str):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    from alien_b200 import abi, dist
    from oracle import oracle as O

    try:
        w, r, _ = dist.init("gloo", timeout_s=20)
        assert (w, r) == (world, rank)
        P = abi.diffusion(10, 10, 10, sigma=1.0, smooth=2.0, seed=rank)
        dist.barrier(w)
        if mode == "fail" and rank == 1:
            raise RuntimeError("rank 1 fails between steps")
        res = O.solve(P.row_ptr, P.cols, P.vals, P.b, solver="cg", precond="diag", tol=1e-8, max_iter=500)
        t = float(res.iterations) + 0.5 * rank  # stands in for the rank's step time
        tmax = dist.reduce_max(w, t)
        total = dist.reduce_sum(w, 1.0)
        dist.barrier(w)
        out.put((rank, res.iterations, bool(res.converged), tmax, total, float(P.vals.sum())))
        dist.finish(w)
    except Exception as e:  # reported to the parent, never a hang
        out.put((rank, "error", type(e).__name__))


def _run(mode: str, world: int = 2):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q, mode)) for r in range(world)]
    for p in procs:
        p.start()
    results = [q.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        if p.is_alive():
            p.kill()
    return sorted(results, key=lambda r: r[0])


def test_two_ranks_independent_systems():
    res = _run("ok")
    assert [r[0] for r in res] == [0, 1]
    iters = [r[1] for r in res]
    assert all(r[2] for r in res)
    assert res[0][3] == res[1][3] == max(iters[0], iters[1] + 0.5)  # max over ranks, seen by every rank
    assert res[0][4] == res[1][4] == 2.0  # systems solved in the job
    assert res[0][5] != res[1][5]  # each rank its own seeded system


def test_rank_failure_is_an_error_not_a_hang():
    res = _run("fail")
    assert res[1][1] == "error"
    assert res[0][1] == "error"  # the survivor's collective ends with an error (timeout / closed peer)
