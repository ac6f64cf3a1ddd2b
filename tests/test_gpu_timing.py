"""Phase timers: device time of every ABI operation by the reference's phase
names (StdTimer sentries, "CSR-SPMV", "CSR-DOT", ...), resolved only when read;
AB2_PERF_TIMER=1 prints them when the context goes, as the reference's
ALIEN_USE_PERF_TIMER build prints its timers."""
import os
import subprocess
import sys

import numpy as np
import pytest

from alien_b200 import abi
from tests import problems

pytestmark = pytest.mark.gpu


def test_phase_times_count_every_call():
    P = problems.get("diffusion12")
    c = abi.Context(0)
    assert c.phase_times() == {}
    A = c.matrix(P.row_ptr, P.cols, P.vals)
    x, y = c.vector(P.b), c.vector(P.n)
    c.set_phase_timing(True)
    for _ in range(3):
        c.mult(A, x, y)
    c.dot(x, y)
    c.dot(y, y)
    c.axpy(0.5, x, y)
    M = abi.Precond(c, A, "ilu0")
    M.apply(x, y)
    S = abi.Solver(c, A, solver="cg", precond="diag", tol=1e-8, max_iter=200)
    S.solve(x, y)
    t = c.phase_times()
    assert t["CSR-SPMV"][0] == 3 and t["CSR-DOT"][0] == 2 and t["CSR-AXPY"][0] == 1
    assert t["PRECOND-ILU0"][0] == 1 and t["SOLVER-CG"][0] == 1
    assert all(ms > 0 for _, ms in t.values())
    assert t["SOLVER-CG"][1] > t["CSR-SPMV"][1] / 3
    c.set_phase_timing(False)
    c.mult(A, x, y)
    assert c.phase_times() == {}
    for o in (S, M, A, x, y, c):
        o.close()


def test_env_prints_phases_when_the_context_goes():
    code = ("import numpy as np\n"
            "from alien_b200 import abi\n"
            "P = abi.poisson(8, 8, 8, seed=0)\n"
            "c = abi.Context(0)\n"
            "A = c.matrix(P.row_ptr, P.cols, P.vals)\n"
            "x, y = c.vector(P.b), c.vector(P.n)\n"
            "c.mult(A, x, y); c.dot(x, y)\n"
            "for o in (A, x, y, c): o.close()\n")
    env = dict(os.environ, AB2_PERF_TIMER="1", PYTHONPATH=str(os.getcwd()))
    out = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, env=env, timeout=300)
    assert out.returncode == 0, out.stderr
    assert "PERF INFO : B200-ALGEBRA" in out.stderr
    assert "CSR-SPMV:" in out.stderr and "CSR-DOT:" in out.stderr
