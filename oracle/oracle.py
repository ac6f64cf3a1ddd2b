"""CPU oracle loader -- TEST INFRASTRUCTURE ONLY.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline legs import
this module.  It wraps two shared libraries built by oracle/Makefile:

* ``_build/libab2_oracle.so`` -- this repo's sequential restatement of Alien's
  SimpleCSR algebra and Krylov templates (ab2_oracle.cpp, citations there);
* ``_ref/libalien_ref.so`` -- Alien's OWN header-only Krylov templates
  (CG.h, BiCGStab.h, Iteration.h, Diag/ILU0/Chebyshev preconditioners)
  compiled from the reference sources over a SimpleCSR-restating CPU algebra
  (ref/ref_driver.cpp).  It pins the restatement: the tests require both to
  agree result for result.
"""
from __future__ import annotations

import ctypes as C
import subprocess
from dataclasses import dataclass
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ORACLE_SO = HERE / "_build" / "libab2_oracle.so"
THREADS_SO = HERE / "_build" / "libab2_oracle_threads.so"  # the same restatement on all host threads
REF_SO = HERE / "_ref" / "libalien_ref.so"

SOLVER = {"cg": 0, "bicgs": 1, "bicgstab": 1}
PRECOND = {"none": 0, "diag": 1, "ilu0": 2, "cheb": 3, "filu0": 4, "neumann": 5}
BREAKDOWN = {0: None, 1: "alpha", 2: "beta", 3: "rho", 9: "other"}


class Options(C.Structure):
    # The reference driver ignores dot_mode, tree_blocks and cheb_lanczos.
    _fields_ = [("solver", C.c_int), ("precond", C.c_int), ("tol", C.c_double), ("max_iter", C.c_int),
                ("poly_factor", C.c_double), ("poly_order", C.c_int), ("poly_factor_max_iter", C.c_int),
                ("dot_mode", C.c_int), ("tree_blocks", C.c_int), ("cheb_saad", C.c_int),
                ("cheb_lanczos", C.c_int), ("filu_factor_iter", C.c_int), ("filu_solver_iter", C.c_int)]


DOT_SEQUENTIAL, DOT_DEVICE_TREE = 0, 1


class Result(C.Structure):
    _fields_ = [("iterations", C.c_int), ("converged", C.c_int), ("error", C.c_int), ("breakdown", C.c_int),
                ("nrm2_b", C.c_double), ("last_rr", C.c_double), ("cheb_alpha", C.c_double),
                ("cheb_beta", C.c_double), ("history_len", C.c_int)]


class MixedOptions(C.Structure):
    _fields_ = [("solver", C.c_int), ("precond", C.c_int), ("tol", C.c_double), ("max_outer", C.c_int),
                ("inner_tol", C.c_double), ("inner_max_iter", C.c_int), ("poly_factor", C.c_double),
                ("poly_order", C.c_int), ("poly_factor_max_iter", C.c_int), ("cheb_saad", C.c_int),
                ("cheb_lanczos", C.c_int), ("dot_mode", C.c_int), ("tree_blocks", C.c_int),
                ("filu_factor_iter", C.c_int), ("filu_solver_iter", C.c_int), ("jacobi_scaled", C.c_int)]


class MixedResult(C.Structure):
    _fields_ = [("succeeded", C.c_int), ("outer_iterations", C.c_int), ("inner_iterations", C.c_int),
                ("error", C.c_int), ("true_residual", C.c_double), ("history_len", C.c_int)]


_DP = C.POINTER(C.c_double)
_IP = C.POINTER(C.c_int)
_FP = C.POINTER(C.c_float)


def build() -> None:
    """Builds the oracle (and the reference-template library when the
    reference sources are present)."""
    subprocess.run(["make", "-s", "-f", str(HERE / "Makefile")], check=True)


def _load(path: Path, prefix: str) -> C.CDLL:
    if not path.exists():
        raise ImportError(f"{path} missing: run make -f oracle/Makefile")
    L = C.CDLL(str(path))
    f = getattr(L, f"{prefix}_solve")
    f.restype = C.c_int
    f.argtypes = [C.c_int, _IP, _IP, _DP, _DP, _DP, C.POINTER(Options), C.POINTER(Result), _DP, C.c_int]
    for name in ("ilu0_factor",):
        g = getattr(L, f"{prefix}_{name}")
        g.restype = C.c_int
        g.argtypes = [C.c_int, _IP, _IP, _DP, _DP]
    g = getattr(L, f"{prefix}_ilu0_apply")
    g.restype = C.c_int
    g.argtypes = [C.c_int, _IP, _IP, _DP, _DP, _DP]
    g = getattr(L, f"{prefix}_cheb_apply")
    g.restype = C.c_int
    g.argtypes = [C.c_int, _IP, _IP, _DP, C.c_double, C.c_int, C.c_int, _DP, _DP]
    g = getattr(L, f"{prefix}_filu0_apply")
    g.restype = C.c_int
    g.argtypes = [C.c_int, _IP, _IP, _DP, C.c_int, C.c_int, _DP, _DP, _DP]
    g = getattr(L, f"{prefix}_neumann_apply")
    g.restype = C.c_int
    g.argtypes = [C.c_int, _IP, _IP, _DP, C.c_double, C.c_int, C.c_int, _DP, _DP, _DP]
    return L


_orc = None
_ref = None


def orc() -> C.CDLL:
    global _orc
    if _orc is None:
        L = _load(ORACLE_SO, "orc")
        L.orc_spmv.argtypes = [C.c_int, _IP, _IP, _DP, _DP, _DP]
        L.orc_add_lmult.argtypes = [C.c_int, _IP, _IP, _DP, C.c_double, _DP, _DP]
        L.orc_add_umult.argtypes = [C.c_int, _IP, _IP, _DP, C.c_double, _DP, _DP]
        L.orc_diag_offsets.argtypes = [C.c_int, _IP, _IP, _IP]
        L.orc_inv_diag.argtypes = [C.c_int, _IP, _IP, _DP, _DP]
        L.orc_dot.argtypes = [C.c_int, _DP, _DP]
        L.orc_dot.restype = C.c_double
        L.orc_dot_tree.argtypes = [C.c_int, _DP, _DP, C.c_int]
        L.orc_dot_tree.restype = C.c_double
        L.orc_set_dot_mode.argtypes = [C.c_int, C.c_int]
        L.orc_set_cheb_variant.argtypes = [C.c_int, C.c_int]
        L.orc_axpy.argtypes = [C.c_int, C.c_double, _DP, _DP]
        L.orc_aypx.argtypes = [C.c_int, C.c_double, _DP, _DP]
        L.orc_cheb_bounds.argtypes = [C.c_int, _IP, _IP, _DP, C.c_double, C.c_int, _DP, _DP]
        L.orc_ell_layout.argtypes = [C.c_int, _IP, _IP, _DP, C.c_int, _IP, _IP, _DP]
        L.orc_spmv32.argtypes = [C.c_int, _IP, _IP, _FP, _FP, _FP]
        L.orc_dot_tree32.argtypes = [C.c_int, _FP, _FP, C.c_int]
        L.orc_dot_tree32.restype = C.c_float
        L.orc_ilu0_apply32.argtypes = [C.c_int, _IP, _IP, _DP, _FP, _FP]
        L.orc_cheb_apply32.argtypes = [C.c_int, _IP, _IP, _DP, _FP, C.c_double, C.c_int, C.c_int, _FP, _FP]
        L.orc_batch_solve.argtypes = [C.c_int, _IP, _IP, _DP, C.c_int, _IP, _DP, _DP, C.c_double, C.c_int,
                                      C.c_double, C.c_int, C.c_int, C.c_int, C.c_int, _IP, _IP, _IP, _DP]
        L.orc_mixed_solve.argtypes = [C.c_int, _IP, _IP, _DP, _DP, _DP, C.POINTER(MixedOptions),
                                      C.POINTER(MixedResult), _DP, C.c_int]
        L.orc_dist_layout.argtypes = [C.c_int, _IP, _IP, _DP, C.c_int, _IP, C.c_int, _IP, _IP, _IP, _DP, _IP, _IP, _IP]
        L.orc_dist_spmv.argtypes = [C.c_int, _IP, _IP, _DP, C.c_int, _IP, _DP, _DP]
        L.orc_dist_dot.argtypes = [C.c_int, _IP, _DP, _DP, C.c_int, C.c_int]
        L.orc_dist_dot.restype = C.c_double
        L.orc_bj_ilu0_apply.argtypes = [C.c_int, _IP, _IP, _DP, C.c_int, _IP, _DP, _DP, _DP]
        L.orc_dist_solve.argtypes = [C.c_int, _IP, _IP, _DP, C.c_int, _IP, _DP, _DP, C.POINTER(Options),
                                     C.POINTER(Result), _DP, C.c_int]
        _orc = L
    return _orc


_thr = None


def threads() -> C.CDLL:
    """The restatement built with its SpMV and BLAS-1 loops on all host
    threads (AB2_CPU_THREADS, default all): the all-cores CPU timing
    baseline -- a restatement, not the reference (its dots sum per-thread
    partials)."""
    global _thr
    if _thr is None:
        _thr = _load(THREADS_SO, "orc")
    return _thr


def ref_available() -> bool:
    return REF_SO.exists()


def ref() -> C.CDLL:
    global _ref
    if _ref is None:
        _ref = _load(REF_SO, "ref")
        _ref.ref_set_cheb_saad.argtypes = [C.c_int]
        _ref.ref_bj_ilu0_apply.argtypes = [C.c_int, C.c_int, _IP, _IP, _DP, _IP, _DP, _DP, _DP]
    return _ref


def _c(a, dt):
    return np.ascontiguousarray(a, dtype=dt)


def _dp(a):
    return a.ctypes.data_as(_DP)


def _ip(a):
    return a.ctypes.data_as(_IP)


def _fp(a):
    return a.ctypes.data_as(_FP)


@dataclass
class OracleSolve:
    x: np.ndarray
    iterations: int
    converged: bool
    error: int
    breakdown: str | None
    nrm2_b: float
    last_rr: float
    cheb_alpha: float
    cheb_beta: float
    history: np.ndarray

    @property
    def residual(self) -> float:
        return float(np.sqrt(self.last_rr / self.nrm2_b)) if self.nrm2_b > 0 else 0.0


def solve(row_ptr, cols, vals, b, x0=None, solver="cg", precond="diag", tol=1e-8, max_iter=1000, poly_factor=0.0,
          poly_order=3, poly_factor_max_iter=10, which="oracle", dot_mode=DOT_SEQUENTIAL,
          tree_blocks=1184, cheb_saad=False, cheb_lanczos=False, filu_factor_iter=0,
          filu_solver_iter=3) -> OracleSolve:
    """Runs the restatement (which='oracle'), the reference templates
    (which='ref') or the restatement on all host threads (which='threads',
    timing only).
    dot_mode=DOT_DEVICE_TREE makes the restatement sum every dot product in
    libab2's reduction tree (tree_blocks = its block cap), for bit-exact checks.
    cheb_saad selects ChebyshevPreconditioner<.., true>; cheb_lanczos (oracle
    only: no reference counterpart) takes the bounds from Lanczos steps."""
    rp, ci, v, bb = _c(row_ptr, np.int32), _c(cols, np.int32), _c(vals, np.float64), _c(b, np.float64)
    n = rp.size - 1
    x = np.zeros(n) if x0 is None else _c(x0, np.float64).copy()
    o = Options(SOLVER[solver], PRECOND[precond], tol, max_iter, poly_factor, poly_order, poly_factor_max_iter,
                dot_mode, tree_blocks, int(cheb_saad), int(cheb_lanczos), filu_factor_iter, filu_solver_iter)
    r = Result()
    cap = 2 * max_iter + 8
    hist = np.zeros(cap)
    L = {"oracle": orc, "ref": ref, "threads": threads}[which]()
    fn = L.ref_solve if which == "ref" else L.orc_solve
    fn(n, _ip(rp), _ip(ci), _dp(v), _dp(bb), _dp(x), C.byref(o), C.byref(r), _dp(hist), cap)
    return OracleSolve(x, r.iterations, bool(r.converged), r.error, BREAKDOWN.get(r.breakdown), r.nrm2_b, r.last_rr,
                       r.cheb_alpha, r.cheb_beta, hist[:min(r.history_len, cap)].copy())


def filu0_apply(row_ptr, cols, vals, y, factor_iter=0, solver_iter=3, which="oracle"):
    """One FILU0 application x = M^-1 y (FILU0Preconditioner.h, the
    device-algebra branch) and the factor in CSR order."""
    rp, ci, v, yy = _c(row_ptr, np.int32), _c(cols, np.int32), _c(vals, np.float64), _c(y, np.float64)
    n = rp.size - 1
    x = np.zeros(n)
    lu = np.zeros(rp[-1])
    L = orc() if which == "oracle" else ref()
    fn = L.orc_filu0_apply if which == "oracle" else L.ref_filu0_apply
    fn(n, _ip(rp), _ip(ci), _dp(v), factor_iter, solver_iter, _dp(yy), _dp(x), _dp(lu))
    return x, lu


def neumann_apply(row_ptr, cols, vals, x, factor, order=3, max_iter=10, which="oracle"):
    """One Neumann-polynomial application y = M^-1 x and the omega used
    (factor = 0: power method; the reference seeds it from random_device)."""
    rp, ci, v, xx = _c(row_ptr, np.int32), _c(cols, np.int32), _c(vals, np.float64), _c(x, np.float64)
    n = rp.size - 1
    y = np.zeros(n)
    om = np.zeros(1)
    L = orc() if which == "oracle" else ref()
    fn = L.orc_neumann_apply if which == "oracle" else L.ref_neumann_apply
    fn(n, _ip(rp), _ip(ci), _dp(v), factor, order, max_iter, _dp(xx), _dp(y), _dp(om))
    return y, float(om[0])


def spmv(row_ptr, cols, vals, x) -> np.ndarray:
    rp, ci, v, xx = _c(row_ptr, np.int32), _c(cols, np.int32), _c(vals, np.float64), _c(x, np.float64)
    y = np.empty(rp.size - 1)
    orc().orc_spmv(rp.size - 1, _ip(rp), _ip(ci), _dp(v), _dp(xx), _dp(y))
    return y


def add_lu_mult(row_ptr, cols, vals, alpha, x, y, lower: bool) -> np.ndarray:
    rp, ci, v, xx = _c(row_ptr, np.int32), _c(cols, np.int32), _c(vals, np.float64), _c(x, np.float64)
    yy = _c(y, np.float64).copy()
    f = orc().orc_add_lmult if lower else orc().orc_add_umult
    f(rp.size - 1, _ip(rp), _ip(ci), _dp(v), alpha, _dp(xx), _dp(yy))
    return yy


def inv_diag(row_ptr, cols, vals) -> np.ndarray:
    rp, ci, v = _c(row_ptr, np.int32), _c(cols, np.int32), _c(vals, np.float64)
    out = np.empty(rp.size - 1)
    orc().orc_inv_diag(rp.size - 1, _ip(rp), _ip(ci), _dp(v), _dp(out))
    return out


def dot(x, y) -> float:
    xx, yy = _c(x, np.float64), _c(y, np.float64)
    return orc().orc_dot(xx.size, _dp(xx), _dp(yy))


def dot_tree(x, y, tree_blocks: int) -> float:
    """x.y summed in libab2's device reduction tree."""
    xx, yy = _c(x, np.float64), _c(y, np.float64)
    return orc().orc_dot_tree(xx.size, _dp(xx), _dp(yy), tree_blocks)


def set_dot_mode(mode: int, tree_blocks: int = 1184) -> None:
    """Dot order for the Chebyshev helpers below (solve() takes it as options)."""
    orc().orc_set_dot_mode(mode, tree_blocks)


def axpy(a, x, y) -> np.ndarray:
    """y + a x with one fma per element (cblas_daxpy)."""
    xx, yy = _c(x, np.float64), _c(y, np.float64).copy()
    orc().orc_axpy(xx.size, a, _dp(xx), _dp(yy))
    return yy


def aypx(a, y, x) -> np.ndarray:
    xx, yy = _c(x, np.float64), _c(y, np.float64).copy()
    orc().orc_aypx(xx.size, a, _dp(yy), _dp(xx))
    return yy


def ilu0_factor(row_ptr, cols, vals, which="oracle") -> np.ndarray:
    rp, ci, v = _c(row_ptr, np.int32), _c(cols, np.int32), _c(vals, np.float64)
    out = np.empty(v.size)
    L = orc() if which == "oracle" else ref()
    getattr(L, "orc_ilu0_factor" if which == "oracle" else "ref_ilu0_factor")(rp.size - 1, _ip(rp), _ip(ci), _dp(v),
                                                                                _dp(out))
    return out


def ilu0_apply(row_ptr, cols, vals, y, which="oracle") -> np.ndarray:
    rp, ci, v, yy = _c(row_ptr, np.int32), _c(cols, np.int32), _c(vals, np.float64), _c(y, np.float64)
    out = np.empty(rp.size - 1)
    L = orc() if which == "oracle" else ref()
    getattr(L, "orc_ilu0_apply" if which == "oracle" else "ref_ilu0_apply")(rp.size - 1, _ip(rp), _ip(ci), _dp(v),
                                                                              _dp(yy), _dp(out))
    return out


def cheb_apply(row_ptr, cols, vals, x, factor=0.0, order=3, max_iter=10, which="oracle", dot_mode=DOT_SEQUENTIAL,
               tree_blocks=1184, saad=False, lanczos=False) -> np.ndarray:
    rp, ci, v, xx = _c(row_ptr, np.int32), _c(cols, np.int32), _c(vals, np.float64), _c(x, np.float64)
    out = np.empty(rp.size - 1)
    set_dot_mode(dot_mode, tree_blocks)
    orc().orc_set_cheb_variant(int(saad), int(lanczos))
    if which != "oracle":
        ref().ref_set_cheb_saad(int(saad))
    L = orc() if which == "oracle" else ref()
    getattr(L, "orc_cheb_apply" if which == "oracle" else "ref_cheb_apply")(rp.size - 1, _ip(rp), _ip(ci), _dp(v),
                                                                              factor, order, max_iter, _dp(xx),
                                                                              _dp(out))
    return out


def cheb_bounds(row_ptr, cols, vals, factor=0.0, max_iter=10, dot_mode=DOT_SEQUENTIAL,
                tree_blocks=1184, lanczos=False) -> tuple[float, float]:
    rp, ci, v = _c(row_ptr, np.int32), _c(cols, np.int32), _c(vals, np.float64)
    a, b = C.c_double(), C.c_double()
    set_dot_mode(dot_mode, tree_blocks)
    orc().orc_set_cheb_variant(0, int(lanczos))
    orc().orc_cheb_bounds(rp.size - 1, _ip(rp), _ip(ci), _dp(v), factor, max_iter, C.byref(a), C.byref(b))
    return a.value, b.value


def ell_layout(row_ptr, cols, vals, slice_rows=32):
    rp, ci, v = _c(row_ptr, np.int32), _c(cols, np.int32), _c(vals, np.float64)
    n = rp.size - 1
    ns = (n + slice_rows - 1) // slice_rows
    off = np.empty(ns + 1, dtype=np.int32)
    orc().orc_ell_layout(n, _ip(rp), _ip(ci), _dp(v), slice_rows, _ip(off), None, None)
    stored = int(off[-1]) * slice_rows
    ec = np.empty(stored, dtype=np.int32)
    ev = np.empty(stored)
    orc().orc_ell_layout(n, _ip(rp), _ip(ci), _dp(v), slice_rows, _ip(off), _ip(ec), _dp(ev))
    return off, ec, ev


# ---------------------------------------------------------------- FP32 / mixed precision
# No reference counterpart: the reference's arithmetic instantiated in float
# (values rounded from FP64; preconditioner set-up in FP64, then rounded).

def spmv32(row_ptr, cols, vals, x) -> np.ndarray:
    rp, ci = _c(row_ptr, np.int32), _c(cols, np.int32)
    v32, xx = _c(np.asarray(vals, np.float64).astype(np.float32), np.float32), _c(x, np.float32)
    y = np.empty(rp.size - 1, dtype=np.float32)
    orc().orc_spmv32(rp.size - 1, _ip(rp), _ip(ci), _fp(v32), _fp(xx), _fp(y))
    return y


def dot_tree32(x, y, tree_blocks: int) -> np.float32:
    xx, yy = _c(x, np.float32), _c(y, np.float32)
    return np.float32(orc().orc_dot_tree32(xx.size, _fp(xx), _fp(yy), tree_blocks))


def ilu0_apply32(row_ptr, cols, vals, y) -> np.ndarray:
    rp, ci, v, yy = _c(row_ptr, np.int32), _c(cols, np.int32), _c(vals, np.float64), _c(y, np.float32)
    out = np.empty(rp.size - 1, dtype=np.float32)
    orc().orc_ilu0_apply32(rp.size - 1, _ip(rp), _ip(ci), _dp(v), _fp(yy), _fp(out))
    return out


def cheb_apply32(row_ptr, cols, vals, x, factor=0.0, order=3, max_iter=10, dot_mode=DOT_SEQUENTIAL,
                 tree_blocks=1184, saad=False, lanczos=False) -> np.ndarray:
    rp, ci, v = _c(row_ptr, np.int32), _c(cols, np.int32), _c(vals, np.float64)
    v32, xx = _c(v.astype(np.float32), np.float32), _c(x, np.float32)
    out = np.empty(rp.size - 1, dtype=np.float32)
    set_dot_mode(dot_mode, tree_blocks)
    orc().orc_set_cheb_variant(int(saad), int(lanczos))
    orc().orc_cheb_apply32(rp.size - 1, _ip(rp), _ip(ci), _dp(v), _fp(v32), factor, order, max_iter, _fp(xx),
                           _fp(out))
    return out


@dataclass
class MixedSolve:
    x: np.ndarray
    succeeded: bool
    outer_iterations: int
    inner_iterations: int
    error: int
    true_residual: float
    history: np.ndarray


def mixed_solve(row_ptr, cols, vals, b, x0=None, solver="cg", precond="diag", tol=1e-8, max_outer=20,
                inner_tol=1e-4, inner_max_iter=1000, poly_factor=0.0, poly_order=3, poly_factor_max_iter=20,
                cheb_saad=False, cheb_lanczos=False, dot_mode=DOT_SEQUENTIAL, tree_blocks=1184, filu_factor_iter=0,
                filu_solver_iter=3, jacobi_scaled=False) -> MixedSolve:
    """FP32 inner Krylov in FP64 refinement, as libab2's ab2_mixed_solve
    (jacobi_scaled: CG + Diag in its symmetrically scaled form)."""
    rp, ci, v, bb = _c(row_ptr, np.int32), _c(cols, np.int32), _c(vals, np.float64), _c(b, np.float64)
    n = rp.size - 1
    x = np.zeros(n) if x0 is None else _c(x0, np.float64).copy()
    o = MixedOptions(SOLVER[solver], PRECOND[precond], tol, max_outer, inner_tol, inner_max_iter, poly_factor,
                     poly_order, poly_factor_max_iter, int(cheb_saad), int(cheb_lanczos), dot_mode, tree_blocks,
                     filu_factor_iter, filu_solver_iter, int(jacobi_scaled))
    r = MixedResult()
    cap = max_outer + 2
    hist = np.zeros(cap)
    orc().orc_mixed_solve(n, _ip(rp), _ip(ci), _dp(v), _dp(bb), _dp(x), C.byref(o), C.byref(r), _dp(hist), cap)
    return MixedSolve(x, bool(r.succeeded), r.outer_iterations, r.inner_iterations, r.error, r.true_residual,
                      hist[:min(r.history_len, cap)].copy())


@dataclass
class BatchSolve:
    x: np.ndarray
    converged: np.ndarray
    outer: np.ndarray
    inner: np.ndarray
    residual: np.ndarray


def batch_solve(row_ptr, cols, vals, sys_offsets, b, x0=None, tol=1e-8, max_outer=20, inner_tol=1e-4,
                inner_max_iter=5000, cluster_size=4, threads=256, lanes_per_row=1) -> BatchSolve:
    """libab2's batched solver restated for a given cluster size, CTA width
    and (CSR) lanes per row: each fixes a reduction tree, hence the rounding.
    The ELL slice width changes nothing (the row sum keeps column order)."""
    rp, ci, v, bb = _c(row_ptr, np.int32), _c(cols, np.int32), _c(vals, np.float64), _c(b, np.float64)
    off = _c(sys_offsets, np.int32)
    n, ns = rp.size - 1, off.size - 1
    x = np.zeros(n) if x0 is None else _c(x0, np.float64).copy()
    conv, outer, inner = (np.zeros(ns, dtype=np.int32) for _ in range(3))
    res = np.zeros(ns)
    orc().orc_batch_solve(n, _ip(rp), _ip(ci), _dp(v), ns, _ip(off), _dp(bb), _dp(x), tol, max_outer, inner_tol,
                          inner_max_iter, cluster_size, threads, lanes_per_row, _ip(conv), _ip(outer), _ip(inner),
                          _dp(res))
    return BatchSolve(x, conv.astype(bool), outer, inner, res)


# ---------------------------------------------------------------------------- row-block distribution
def dist_layout(row_ptr, cols, vals, offsets, rank) -> dict:
    """One rank's rows in the reference's distributed layout (DistStructInfo)."""
    rp, ci, v, off = _c(row_ptr, np.int32), _c(cols, np.int32), _c(vals, np.float64), _c(offsets, np.int32)
    n, k = rp.size - 1, off.size - 1
    sz = np.zeros(4, np.int32)
    orc().orc_dist_layout(n, _ip(rp), _ip(ci), _dp(v), k, _ip(off), rank, _ip(sz), None, None, None, None, None, None)
    nl, ng, ni, nnz = (int(t) for t in sz)
    out = dict(row_ptr=np.empty(nl + 1, np.int32), cols=np.empty(nnz, np.int32), vals=np.empty(nnz),
               local_row_size=np.empty(nl, np.int32), ghost_uids=np.empty(ng, np.int32),
               interface_rows=np.empty(ni, np.int32))
    orc().orc_dist_layout(n, _ip(rp), _ip(ci), _dp(v), k, _ip(off), rank, _ip(sz), _ip(out["row_ptr"]),
                          _ip(out["cols"]), _dp(out["vals"]), _ip(out["local_row_size"]), _ip(out["ghost_uids"]),
                          _ip(out["interface_rows"]))
    return out


def dist_spmv(row_ptr, cols, vals, offsets, x) -> np.ndarray:
    rp, ci, v, off, xx = _c(row_ptr, np.int32), _c(cols, np.int32), _c(vals, np.float64), _c(offsets, np.int32), \
        _c(x, np.float64)
    y = np.empty(rp.size - 1)
    orc().orc_dist_spmv(rp.size - 1, _ip(rp), _ip(ci), _dp(v), off.size - 1, _ip(off), _dp(xx), _dp(y))
    return y


def dist_dot(offsets, x, y, dot_mode=DOT_SEQUENTIAL, tree_blocks=1184) -> float:
    off, xx, yy = _c(offsets, np.int32), _c(x, np.float64), _c(y, np.float64)
    return orc().orc_dist_dot(off.size - 1, _ip(off), _dp(xx), _dp(yy), dot_mode, tree_blocks)


def bj_ilu0_apply(row_ptr, cols, vals, offsets, y):
    """Block-Jacobi ILU(0) over the row blocks: (x, per-rank factors on their local entries)."""
    rp, ci, v, off, yy = _c(row_ptr, np.int32), _c(cols, np.int32), _c(vals, np.float64), _c(offsets, np.int32), \
        _c(y, np.float64)
    n = rp.size - 1
    x = np.empty(n)
    lu = np.empty(ci.size)
    orc().orc_bj_ilu0_apply(n, _ip(rp), _ip(ci), _dp(v), off.size - 1, _ip(off), _dp(yy), _dp(x), _dp(lu))
    # split per rank: each rank's local entries
    parts, o = [], 0
    for r in range(off.size - 1):
        L = dist_layout(rp, ci, v, off, r)
        m = int(L["local_row_size"].sum())
        parts.append(lu[o:o + m].copy())
        o += m
    return x, parts


def ref_bj_ilu0_apply(layout: dict, y):
    """The reference's parallel LUFactorisationAlgo on one rank's layout: (x, factor in distributed order)."""
    rp, ci, v, lrs = (_c(layout[k], dt) for k, dt in (("row_ptr", np.int32), ("cols", np.int32),
                                                        ("vals", np.float64), ("local_row_size", np.int32)))
    n = rp.size - 1
    yy = _c(y, np.float64)
    x = np.empty(n)
    lu = np.empty(ci.size)
    ref().ref_bj_ilu0_apply(n, int(layout["ghost_uids"].size), _ip(rp), _ip(ci), _dp(v), _ip(lrs), _dp(yy), _dp(x),
                            _dp(lu))
    return x, lu


def dist_solve(row_ptr, cols, vals, offsets, b, x0=None, solver="cg", precond="diag", tol=1e-8, max_iter=1000,
               dot_mode=DOT_SEQUENTIAL, tree_blocks=1184) -> OracleSolve:
    """The solve every rank runs on the distributed algebra (block-Jacobi ILU0,
    dots summed over the ranks in rank order)."""
    rp, ci, v, bb, off = _c(row_ptr, np.int32), _c(cols, np.int32), _c(vals, np.float64), _c(b, np.float64), \
        _c(offsets, np.int32)
    n = rp.size - 1
    x = np.zeros(n) if x0 is None else _c(x0, np.float64).copy()
    o = Options(SOLVER[solver], PRECOND[precond], tol, max_iter, 0.0, 3, 10, dot_mode, tree_blocks, 0, 0, 0, 3)
    r = Result()
    cap = 2 * max_iter + 8
    hist = np.zeros(cap)
    orc().orc_dist_solve(n, _ip(rp), _ip(ci), _dp(v), off.size - 1, _ip(off), _dp(bb), _dp(x), C.byref(o), C.byref(r),
                         _dp(hist), cap)
    return OracleSolve(x, r.iterations, bool(r.converged), r.error, BREAKDOWN.get(r.breakdown), r.nrm2_b, r.last_rr,
                       0.0, 0.0, hist[:min(r.history_len, cap)].copy())


# ----------------------------------------------------------------------------- inputs without libab2
INPUTS_SO = HERE / "_build" / "libab2_inputs.so"
_inp = None


class _Problem(C.Structure):
    # struct ab2_problem (include/ab2_problems.h)
    _fields_ = [("n", C.c_int), ("nnz", C.c_longlong), ("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int),
                ("row_ptr", _IP), ("cols", _IP), ("vals", _DP), ("x_true", _DP), ("b", _DP), ("log10_k", _DP)]


@dataclass
class InputProblem:
    """A seeded system as the CPU timing legs see it (same fields as
    alien_b200.abi.CsrProblem)."""
    n: int
    row_ptr: np.ndarray
    cols: np.ndarray
    vals: np.ndarray
    x_true: np.ndarray | None
    b: np.ndarray
    log10_k: np.ndarray | None
    shape: tuple

    @property
    def nnz(self) -> int:
        return int(self.row_ptr[-1])


def inputs() -> C.CDLL:
    """libab2's input generators built for the host alone (oracle/Makefile),
    so that a CPU-only process makes the same system without loading the
    CUDA library."""
    global _inp
    if _inp is None:
        if not INPUTS_SO.exists():
            raise ImportError(f"{INPUTS_SO} missing: run make -f oracle/Makefile")
        L = C.CDLL(str(INPUTS_SO))
        PP = C.POINTER(C.POINTER(_Problem))
        L.ab2_problem_poisson.argtypes = [C.c_int, C.c_int, C.c_int, C.c_uint64, PP]
        L.ab2_problem_diffusion.argtypes = [C.c_int, C.c_int, C.c_int, C.c_double, C.c_double, C.c_uint64, PP]
        L.ab2_problem_convdiff.argtypes = [C.c_int, C.c_int, C.c_int, C.c_double, C.c_int, C.c_uint64, PP]
        L.ab2_problem_destroy.argtypes = [C.POINTER(_Problem)]
        for f in (L.ab2_problem_poisson, L.ab2_problem_diffusion, L.ab2_problem_convdiff, L.ab2_problem_destroy):
            f.restype = C.c_int
        _inp = L
    return _inp


def _take_problem(p) -> InputProblem:
    P = p.contents
    n, nnz = P.n, P.nnz

    def arr(ptr, count, dt):
        return np.ctypeslib.as_array(ptr, shape=(count,)).astype(dt, copy=True)

    out = InputProblem(n, arr(P.row_ptr, n + 1, np.int32), arr(P.cols, nnz, np.int32), arr(P.vals, nnz, np.float64),
                       arr(P.x_true, n, np.float64) if bool(P.x_true) else None, arr(P.b, n, np.float64),
                       arr(P.log10_k, n, np.float64) if bool(P.log10_k) else None, (P.nx, P.ny, P.nz))
    inputs().ab2_problem_destroy(p)
    return out


def problem_poisson(nx, ny=None, nz=None, seed=0) -> InputProblem:
    ny = nx if ny is None else ny
    nz = nx if nz is None else nz
    p = C.POINTER(_Problem)()
    rc = inputs().ab2_problem_poisson(nx, ny, nz, seed, C.byref(p))
    if rc:
        raise RuntimeError(f"ab2_problem_poisson failed ({rc})")
    return _take_problem(p)


def problem_diffusion(nx, ny=None, nz=None, sigma=1.0, smooth=4.0, seed=0) -> InputProblem:
    ny = nx if ny is None else ny
    nz = nx if nz is None else nz
    p = C.POINTER(_Problem)()
    rc = inputs().ab2_problem_diffusion(nx, ny, nz, sigma, smooth, seed, C.byref(p))
    if rc:
        raise RuntimeError(f"ab2_problem_diffusion failed ({rc})")
    return _take_problem(p)


def problem_convdiff(nx, ny=None, nz=None, peclet=10.0, modes=8, seed=0) -> InputProblem:
    ny = nx if ny is None else ny
    nz = nx if nz is None else nz
    p = C.POINTER(_Problem)()
    rc = inputs().ab2_problem_convdiff(nx, ny, nz, peclet, modes, seed, C.byref(p))
    if rc:
        raise RuntimeError(f"ab2_problem_convdiff failed ({rc})")
    return _take_problem(p)
