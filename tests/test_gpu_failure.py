"""Failure detection on the GPU without a fault.

Every device-side wait in libab2 (the sentinel polling of the ILU(0) sweeps)
is bounded by a clock budget and an error flag.  Here one thread waits on a
word that nothing writes -- a producer that is gone: the wait must give up by
itself, set the flag the host reads, and leave the context usable.  (Host-side
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
