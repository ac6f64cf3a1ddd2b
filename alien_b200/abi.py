"""ctypes binding of libab2 (include/ab2.h, include/ab2_dist.h, include/ab2_problems.h).

This is the Python face of the C ABI, shaped like Alien's algebra/solver API
(SimpleCSRInternalLinearAlgebra method names, the krylov example's solver and
preconditioner options, SolverStatus).  It loads ``alien_b200/lib/libab2.so``
and nothing else: when the library is missing the import fails loudly -- there
is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass
from pathlib import Path

import numpy as np

LIB_PATH = Path(os.environ.get("AB2_LIB", Path(__file__).resolve().parent / "lib" / "libab2.so"))

AB2_OK = 0
AB2_ERR_CUDA = -1
AB2_ERR_OOM = -2
AB2_ERR_BREAKDOWN = -3
AB2_ERR_NOT_CONVERGED = -4
AB2_ERR_TIMEOUT = -5
AB2_ERR_BAD_ARG = -6
AB2_ERR_UNSUPPORTED = -7

FMT_CSR, FMT_ELL, FMT_F32, FMT_STENCIL = 1, 2, 4, 8
SPMV_AUTO, SPMV_CSR_SCALAR, SPMV_CSR_STAGED, SPMV_ELL, SPMV_CSR_VECTOR, SPMV_STENCIL = 0, 1, 2, 3, 4, 5
SOLVER = {"cg": 0, "bicgs": 1, "bicgstab": 1}
PRECOND = {"none": 0, "diag": 1, "ilu0": 2, "cheb": 3, "filu0": 4, "neumann": 5}
ILU_SCHEDULE = {"auto": 0, "wavefront": 1, "stencil": 2, "stencil_cluster": 3}
BREAKDOWN = {0: None, 1: "alpha", 2: "beta", 3: "rho"}
FCG_FALLBACK = {"sticky": 0, "step": 1}
GNN_LAYER = {"auto": 0, "gather": 1, "grid": 2}
MIXED_JACOBI = {"auto": 0, "plain": 1, "scaled": 2}
COMM_ID_BYTES = 128


class AB2Error(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"libab2 error {code}: {msg}")
        self.code = code


class ContextInfo(C.Structure):
    _fields_ = [("device", C.c_int), ("num_sms", C.c_int), ("reduction_threads", C.c_int),
                ("reduction_max_blocks", C.c_int)]


class MatrixInfo(C.Structure):
    _fields_ = [("n", C.c_int), ("nnz", C.c_longlong), ("ell_stored", C.c_longlong), ("ell_slice", C.c_int),
                ("formats", C.c_int), ("device_bytes", C.c_longlong), ("stencil_bands", C.c_int),
                ("stencil_nx", C.c_int), ("stencil_ny", C.c_int), ("stencil_nz", C.c_int)]


class PrecondOptions(C.Structure):
    _fields_ = [("kind", C.c_int), ("poly_factor", C.c_double), ("poly_order", C.c_int),
                ("poly_factor_max_iter", C.c_int), ("ilu_schedule", C.c_int), ("cheb_saad", C.c_int),
                ("cheb_lanczos", C.c_int), ("filu_factor_iter", C.c_int), ("filu_solver_iter", C.c_int),
                ("filu_tol", C.c_double)]


class PrecondInfo(C.Structure):
    _fields_ = [("kind", C.c_int), ("cheb_alpha", C.c_double), ("cheb_beta", C.c_double),
                ("ilu_levels_lower", C.c_int), ("ilu_levels_upper", C.c_int), ("ilu_schedule", C.c_int),
                ("neumann_factor", C.c_double)]


class SolverOptions(C.Structure):
    _fields_ = [("solver", C.c_int), ("precond", C.c_int), ("tol", C.c_double), ("max_iter", C.c_int),
                ("poly_factor", C.c_double), ("poly_order", C.c_int), ("poly_factor_max_iter", C.c_int),
                ("spmv_variant", C.c_int), ("use_graph", C.c_int), ("ilu_schedule", C.c_int),
                ("cheb_saad", C.c_int), ("cheb_lanczos", C.c_int), ("filu_factor_iter", C.c_int),
                ("filu_solver_iter", C.c_int), ("filu_tol", C.c_double)]


class Status(C.Structure):
    _fields_ = [("succeeded", C.c_int), ("iterations", C.c_int), ("error", C.c_int), ("breakdown", C.c_int),
                ("residual", C.c_double), ("true_residual", C.c_double), ("nrm2_b", C.c_double),
                ("setup_ms", C.c_double), ("solve_ms", C.c_double)]


class MixedOptions(C.Structure):
    _fields_ = [("solver", C.c_int), ("precond", C.c_int), ("tol", C.c_double), ("max_outer", C.c_int),
                ("inner_tol", C.c_double), ("inner_max_iter", C.c_int), ("poly_factor", C.c_double),
                ("poly_order", C.c_int), ("poly_factor_max_iter", C.c_int), ("cheb_saad", C.c_int),
                ("cheb_lanczos", C.c_int), ("ilu_schedule", C.c_int), ("spmv_variant", C.c_int),
                ("use_graph", C.c_int), ("filu_factor_iter", C.c_int),
                ("filu_solver_iter", C.c_int), ("filu_tol", C.c_double), ("jacobi_form", C.c_int)]


class MixedStatus(C.Structure):
    _fields_ = [("succeeded", C.c_int), ("outer_iterations", C.c_int), ("inner_iterations", C.c_int),
                ("error", C.c_int), ("true_residual", C.c_double), ("setup_ms", C.c_double),
                ("solve_ms", C.c_double), ("jacobi_scaled", C.c_int)]


class BatchOptions(C.Structure):
    _fields_ = [("tol", C.c_double), ("max_outer", C.c_int), ("inner_tol", C.c_double), ("inner_max_iter", C.c_int),
                ("spmv_variant", C.c_int), ("cluster_size", C.c_int), ("threads", C.c_int), ("tune_iters", C.c_int),
                ("ell_slice", C.c_int), ("lanes_per_row", C.c_int)]


class BatchTrial(C.Structure):
    _fields_ = [("spmv_variant", C.c_int), ("cluster_size", C.c_int), ("threads", C.c_int), ("ms", C.c_float),
                ("ell_slice", C.c_int), ("lanes_per_row", C.c_int)]


class BatchInfo(C.Structure):
    _fields_ = [("nsys", C.c_int), ("rows", C.c_longlong), ("spmv_variant", C.c_int), ("cluster_size", C.c_int),
                ("threads", C.c_int), ("tuned", C.c_int), ("tune_ms", C.c_double), ("setup_ms", C.c_double),
                ("trials", C.c_int), ("ell_slice", C.c_int), ("lanes_per_row", C.c_int)]


class BatchStatus(C.Structure):
    _fields_ = [("systems_converged", C.c_int), ("max_outer", C.c_int), ("inner_total", C.c_longlong),
                ("inner_max", C.c_int), ("max_residual", C.c_double), ("solve_ms", C.c_double)]


class FcgOptions(C.Structure):
    _fields_ = [("tol", C.c_double), ("max_iter", C.c_int), ("fallback_ratio", C.c_double), ("truncation", C.c_int),
                ("fallback_mode", C.c_int)]


class FcgStatus(C.Structure):
    _fields_ = [("succeeded", C.c_int), ("iterations", C.c_int), ("gnn_steps", C.c_int), ("fallback_steps", C.c_int),
                ("switched_at", C.c_int), ("error", C.c_int), ("true_residual", C.c_double),
                ("solve_ms", C.c_double)]


class PhaseTime(C.Structure):
    _fields_ = [("name", C.c_char * 32), ("calls", C.c_longlong), ("ms", C.c_double)]


class DistInfo(C.Structure):
    _fields_ = [("global_rows", C.c_int), ("local_rows", C.c_int), ("ghost_rows", C.c_int),
                ("interface_rows", C.c_int), ("recv_neighbours", C.c_int), ("send_neighbours", C.c_int),
                ("send_count", C.c_int), ("first_upper_ghost_index", C.c_int), ("local_nnz", C.c_longlong),
                ("ghost_nnz", C.c_longlong)]


class Problem(C.Structure):
    _fields_ = [("n", C.c_int), ("nnz", C.c_longlong), ("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int),
                ("row_ptr", C.POINTER(C.c_int)), ("cols", C.POINTER(C.c_int)), ("vals", C.POINTER(C.c_double)),
                ("x_true", C.POINTER(C.c_double)), ("b", C.POINTER(C.c_double)),
                ("log10_k", C.POINTER(C.c_double))]


_P = C.c_void_p
_I = C.c_int
_D = C.c_double
_DP = C.POINTER(C.c_double)
_IP = C.POINTER(C.c_int)

# name -> (restype, argtypes); the full list of entry points in include/*.h
SIGNATURES: dict[str, tuple] = {
    "ab2_context_create": (_I, [_I, C.POINTER(_P)]),
    "ab2_context_destroy": (_I, [_P]),
    "ab2_last_error_message": (C.c_char_p, [_P]),
    "ab2_context_stream": (_I, [_P, C.POINTER(_P)]),
    "ab2_synchronize": (_I, [_P]),
    "ab2_context_launch_count": (_I, [_P, C.POINTER(C.c_longlong)]),
    "ab2_context_get_info": (_I, [_P, C.POINTER(ContextInfo)]),
    "ab2_context_set_phase_timing": (_I, [_P, _I]),
    "ab2_context_phase_times": (_I, [_P, C.POINTER(PhaseTime), _I, _IP]),
    "ab2_matrix_create_csr": (_I, [_P, _I, _IP, _IP, _DP, _I, C.POINTER(_P)]),
    "ab2_matrix_update_values": (_I, [_P, _P, _DP]),
    "ab2_matrix_destroy": (_I, [_P]),
    "ab2_matrix_get_info": (_I, [_P, C.POINTER(MatrixInfo)]),
    "ab2_vector_create": (_I, [_P, _I, C.POINTER(_P)]),
    "ab2_vector_destroy": (_I, [_P]),
    "ab2_vector_size": (_I, [_P, _IP]),
    "ab2_vector_upload": (_I, [_P, _P, _DP]),
    "ab2_vector_download": (_I, [_P, _P, _DP]),
    "ab2_vector_device_ptr": (_I, [_P, C.POINTER(_P)]),
    "ab2_mult": (_I, [_P, _P, _P, _P]),
    "ab2_mult_variant": (_I, [_P, _P, _P, _P, _I]),
    "ab2_add_lmult": (_I, [_P, _D, _P, _P, _P]),
    "ab2_add_umult": (_I, [_P, _D, _P, _P, _P]),
    "ab2_compute_inv_diag": (_I, [_P, _P, _P]),
    "ab2_mult_inv_diag": (_I, [_P, _P, _P]),
    "ab2_axpy": (_I, [_P, _D, _P, _P]),
    "ab2_aypx": (_I, [_P, _D, _P, _P]),
    "ab2_copy": (_I, [_P, _P, _P]),
    "ab2_scal": (_I, [_P, _D, _P]),
    "ab2_pointwise_mult": (_I, [_P, _P, _P, _P]),
    "ab2_assign": (_I, [_P, _P, _D]),
    "ab2_diagonal": (_I, [_P, _P, _P]),
    "ab2_reciprocal": (_I, [_P, _P]),
    "ab2_dot": (_I, [_P, _P, _P, _DP]),
    "ab2_norm0": (_I, [_P, _P, _DP]),
    "ab2_norm1": (_I, [_P, _P, _DP]),
    "ab2_norm2": (_I, [_P, _P, _DP]),
    "ab2_scalar_create": (_I, [_P, C.POINTER(_P)]),
    "ab2_scalar_destroy": (_I, [_P]),
    "ab2_dot_async": (_I, [_P, _P, _P, _P]),
    "ab2_scalar_get": (_I, [_P, _P, _DP]),
    "ab2_dot_noalloc": (_I, [_P, _P, _I, _P, _P]),
    "ab2_precond_create": (_I, [_P, _P, C.POINTER(PrecondOptions), C.POINTER(_P)]),
    "ab2_precond_apply": (_I, [_P, _P, _P, _P]),
    "ab2_precond_destroy": (_I, [_P]),
    "ab2_precond_get_info": (_I, [_P, C.POINTER(PrecondInfo)]),
    "ab2_precond_ilu0_values": (_I, [_P, _P, _DP]),
    "ab2_solver_options_default": (None, [C.POINTER(SolverOptions)]),
    "ab2_solver_create": (_I, [_P, _P, C.POINTER(SolverOptions), C.POINTER(_P)]),
    "ab2_solver_solve": (_I, [_P, _P, _P, C.POINTER(Status)]),
    "ab2_solver_history": (_I, [_P, _DP, _I, _IP]),
    "ab2_solver_destroy": (_I, [_P]),
    "ab2_mixed_options_default": (None, [C.POINTER(MixedOptions)]),
    "ab2_mixed_create": (_I, [_P, _P, C.POINTER(MixedOptions), C.POINTER(_P)]),
    "ab2_mixed_solve": (_I, [_P, _P, _P, C.POINTER(MixedStatus)]),
    "ab2_mixed_history": (_I, [_P, _DP, _I, _IP]),
    "ab2_mixed_destroy": (_I, [_P]),
    "ab2_batch_options_default": (None, [C.POINTER(BatchOptions)]),
    "ab2_batch_create": (_I, [_P, _P, _I, _IP, C.POINTER(BatchOptions), C.POINTER(_P)]),
    "ab2_batch_solve": (_I, [_P, _P, _P, C.POINTER(BatchStatus)]),
    "ab2_batch_results": (_I, [_P, _IP, _IP, _IP, _DP]),
    "ab2_batch_get_info": (_I, [_P, C.POINTER(BatchInfo)]),
    "ab2_batch_trials": (_I, [_P, C.POINTER(BatchTrial), _I]),
    "ab2_batch_destroy": (_I, [_P]),
    "ab2_gnn_param_count": (_I, []),
    "ab2_gnn_create": (_I, [_P, C.POINTER(C.c_float), C.c_ulonglong, C.POINTER(_P)]),
    "ab2_gnn_get_params": (_I, [_P, C.POINTER(C.c_float)]),
    "ab2_gnn_set_params": (_I, [_P, C.POINTER(C.c_float)]),
    "ab2_gnn_set_layer": (_I, [_P, _I]),
    "ab2_gnn_get_layer": (_I, [_P, C.POINTER(C.c_int)]),
    "ab2_gnn_bind": (_I, [_P, _P]),
    "ab2_gnn_apply": (_I, [_P, _P, _P]),
    "ab2_gnn_loss_grad": (_I, [_P, _P, _P, _DP, C.POINTER(C.c_float)]),
    "ab2_gnn_train_step": (_I, [_P, _P, _P, _D, _DP]),
    "ab2_gnn_destroy": (_I, [_P]),
    "ab2_fcg_options_default": (None, [C.POINTER(FcgOptions)]),
    "ab2_fcg_solve": (_I, [_P, _P, _P, _P, _P, _P, C.POINTER(FcgOptions), C.POINTER(FcgStatus)]),
    "ab2_comm_local_group": (_I, [C.POINTER(_P), _I, _D, C.POINTER(_P)]),
    "ab2_comm_nccl_unique_id": (_I, [C.POINTER(C.c_ubyte)]),
    "ab2_comm_nccl_create": (_I, [_P, C.POINTER(C.c_ubyte), _I, _I, C.POINTER(_P)]),
    "ab2_comm_rank": (_I, [_P, _IP]),
    "ab2_comm_size": (_I, [_P, _IP]),
    "ab2_comm_destroy": (_I, [_P]),
    "ab2_dist_matrix_create": (_I, [_P, _P, _IP, _IP, _IP, _DP, _I, C.POINTER(_P)]),
    "ab2_dist_matrix_get_info": (_I, [_P, C.POINTER(DistInfo)]),
    "ab2_dist_matrix_layout": (_I, [_P, _IP, _IP, _DP, _IP, _IP, _IP]),
    "ab2_dist_matrix_plan": (_I, [_P, _IP, _IP, _IP, _IP, _IP]),
    "ab2_dist_matrix_local": (_I, [_P, C.POINTER(_P)]),
    "ab2_dist_matrix_destroy": (_I, [_P]),
    "ab2_dist_vector_create": (_I, [_P, _P, C.POINTER(_P)]),
    "ab2_dist_mult": (_I, [_P, _P, _P, _P]),
    "ab2_dist_dot": (_I, [_P, _P, _P, _P, _DP]),
    "ab2_dist_norm1": (_I, [_P, _P, _P, _DP]),
    "ab2_dist_norm2": (_I, [_P, _P, _P, _DP]),
    "ab2_dist_precond_create": (_I, [_P, _P, C.POINTER(PrecondOptions), C.POINTER(_P)]),
    "ab2_dist_solver_create": (_I, [_P, _P, _P, C.POINTER(SolverOptions), C.POINTER(_P)]),
    "ab2_dist_solver_solve": (_I, [_P, _P, _P, C.POINTER(Status)]),
    "ab2_dist_solver_history": (_I, [_P, _DP, _I, _IP]),
    "ab2_dist_solver_destroy": (_I, [_P]),
    "ab2_problem_poisson": (_I, [_I, _I, _I, C.c_uint64, C.POINTER(C.POINTER(Problem))]),
    "ab2_problem_diffusion": (_I, [_I, _I, _I, _D, _D, C.c_uint64, C.POINTER(C.POINTER(Problem))]),
    "ab2_problem_convdiff": (_I, [_I, _I, _I, _D, _I, C.c_uint64, C.POINTER(C.POINTER(Problem))]),
    "ab2_problem_destroy": (_I, [C.POINTER(Problem)]),
    "ab2_problem_read_matrix_market": (_I, [C.c_char_p, C.c_char_p, C.POINTER(C.POINTER(Problem))]),
    "ab2_problem_write_matrix_market": (_I, [C.POINTER(Problem), C.c_char_p, C.c_char_p]),
    "ab2_matrix_market_error": (C.c_char_p, []),
    "ab2_selftest_bounded_wait": (_I, [_P, _IP, _DP]),
    "ab2_selftest_mbarrier_wait": (_I, [_P, _IP, _DP]),
    "ab2_context_inject_alloc_failure": (_I, [_P, C.c_longlong]),
    "ab2_rng_u64": (C.c_uint64, [C.c_uint64, C.c_uint64, C.c_uint64]),
    "ab2_rng_uniform": (_D, [C.c_uint64, C.c_uint64, C.c_uint64]),
}

_lib = None


def lib() -> C.CDLL:
    """The loaded libab2 (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise ImportError(f"libab2 not built: {LIB_PATH} is missing (run python -m alien_b200.build)")
        L = C.CDLL(str(LIB_PATH))
        for name, (res, args) in SIGNATURES.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def _dp(a: np.ndarray):
    return a.ctypes.data_as(_DP)


def _ip(a: np.ndarray):
    return a.ctypes.data_as(_IP)


# ---------------------------------------------------------------------------- handles
class Context:
    """One CUDA device + stream (ab2_context)."""

    def __init__(self, device: int = 0):
        h = _P()
        rc = lib().ab2_context_create(device, C.byref(h))
        if rc != AB2_OK:
            raise AB2Error(rc, "ab2_context_create failed")
        self.h = h

    def check(self, rc: int, what: str = ""):
        if rc != AB2_OK:
            msg = lib().ab2_last_error_message(self.h) or b""
            raise AB2Error(rc, f"{what}: {msg.decode(errors='replace')}")
        return rc

    def close(self):
        if self.h:
            lib().ab2_context_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def synchronize(self):
        self.check(lib().ab2_synchronize(self.h), "synchronize")

    @property
    def stream(self) -> int:
        s = _P()
        self.check(lib().ab2_context_stream(self.h, C.byref(s)))
        return s.value or 0

    @property
    def info(self) -> ContextInfo:
        i = ContextInfo()
        self.check(lib().ab2_context_get_info(self.h, C.byref(i)))
        return i

    @property
    def launches(self) -> int:
        c = C.c_longlong()
        self.check(lib().ab2_context_launch_count(self.h, C.byref(c)))
        return c.value

    def set_phase_timing(self, on: bool = True) -> None:
        """Phase timers on (restarted at zero) or off: device time per ABI operation ("CSR-SPMV", ...)."""
        self.check(lib().ab2_context_set_phase_timing(self.h, int(on)), "set_phase_timing")

    def phase_times(self) -> dict:
        """{phase: (calls, ms)} of the operations since timing was turned on (synchronises)."""
        n = C.c_int()
        self.check(lib().ab2_context_phase_times(self.h, None, 0, C.byref(n)), "phase_times")
        arr = (PhaseTime * max(n.value, 1))()
        self.check(lib().ab2_context_phase_times(self.h, arr, n.value, C.byref(n)), "phase_times")
        return {arr[i].name.decode(): (arr[i].calls, arr[i].ms) for i in range(n.value)}

    def selftest_bounded_wait(self) -> tuple[bool, float]:
        """(expired, seconds): a device-side wait on a word nothing writes gives up on its budget."""
        e, t = C.c_int(), C.c_double()
        self.check(lib().ab2_selftest_bounded_wait(self.h, C.byref(e), C.byref(t)), "selftest_bounded_wait")
        return bool(e.value), t.value

    def selftest_mbarrier_wait(self) -> tuple[bool, float]:
        """(expired, seconds): a wait on an mbarrier phase nothing completes gives up on its budget."""
        e, t = C.c_int(), C.c_double()
        self.check(lib().ab2_selftest_mbarrier_wait(self.h, C.byref(e), C.byref(t)), "selftest_mbarrier_wait")
        return bool(e.value), t.value

    def inject_alloc_failure(self, nth: int) -> None:
        """The nth device allocation from now on fails as AB2_ERR_OOM (0: off)."""
        self.check(lib().ab2_context_inject_alloc_failure(self.h, nth), "inject_alloc_failure")

    # -- objects
    def matrix(self, row_ptr, cols, vals, formats: int = FMT_CSR | FMT_ELL) -> "Matrix":
        return Matrix(self, row_ptr, cols, vals, formats)

    def vector(self, n_or_array) -> "Vector":
        if np.isscalar(n_or_array):
            return Vector(self, int(n_or_array))
        a = np.ascontiguousarray(n_or_array, dtype=np.float64)
        v = Vector(self, a.size)
        v.upload(a)
        return v

    # -- algebra (IInternalLinearAlgebra method names)
    def mult(self, A, x, y, variant: int = SPMV_AUTO):
        self.check(lib().ab2_mult_variant(self.h, A.h, x.h, y.h, variant), "mult")

    def addLMult(self, alpha, A, x, y):
        self.check(lib().ab2_add_lmult(self.h, alpha, A.h, x.h, y.h), "addLMult")

    def addUMult(self, alpha, A, x, y):
        self.check(lib().ab2_add_umult(self.h, alpha, A.h, x.h, y.h), "addUMult")

    def computeInvDiag(self, A, d):
        self.check(lib().ab2_compute_inv_diag(self.h, A.h, d.h), "computeInvDiag")

    def multInvDiag(self, A, y):
        self.check(lib().ab2_mult_inv_diag(self.h, A.h, y.h), "multInvDiag")

    def diagonal(self, A, d):
        self.check(lib().ab2_diagonal(self.h, A.h, d.h), "diagonal")

    def axpy(self, alpha, x, y):
        self.check(lib().ab2_axpy(self.h, alpha, x.h, y.h), "axpy")

    def aypx(self, alpha, y, x):
        self.check(lib().ab2_aypx(self.h, alpha, y.h, x.h), "aypx")

    def copy(self, x, y):
        self.check(lib().ab2_copy(self.h, x.h, y.h), "copy")

    def scal(self, alpha, x):
        self.check(lib().ab2_scal(self.h, alpha, x.h), "scal")

    def pointwiseMult(self, x, y, w):
        self.check(lib().ab2_pointwise_mult(self.h, x.h, y.h, w.h), "pointwiseMult")

    def assign(self, x, alpha):
        self.check(lib().ab2_assign(self.h, x.h, alpha), "assign")

    def reciprocal(self, x):
        self.check(lib().ab2_reciprocal(self.h, x.h), "reciprocal")

    def dot(self, x, y) -> float:
        r = C.c_double()
        self.check(lib().ab2_dot(self.h, x.h, y.h, C.byref(r)), "dot")
        return r.value

    def norm0(self, x) -> float:
        r = C.c_double()
        self.check(lib().ab2_norm0(self.h, x.h, C.byref(r)), "norm0")
        return r.value

    def norm1(self, x) -> float:
        r = C.c_double()
        self.check(lib().ab2_norm1(self.h, x.h, C.byref(r)), "norm1")
        return r.value

    def norm2(self, x) -> float:
        r = C.c_double()
        self.check(lib().ab2_norm2(self.h, x.h, C.byref(r)), "norm2")
        return r.value


class Matrix:
    def __init__(self, ctx: Context, row_ptr, cols, vals, formats: int):
        self.ctx = ctx
        self.row_ptr = np.ascontiguousarray(row_ptr, dtype=np.int32)
        self.cols = np.ascontiguousarray(cols, dtype=np.int32)
        self.vals = np.ascontiguousarray(vals, dtype=np.float64)
        self.n = self.row_ptr.size - 1
        h = _P()
        ctx.check(lib().ab2_matrix_create_csr(ctx.h, self.n, _ip(self.row_ptr), _ip(self.cols), _dp(self.vals),
                                              formats, C.byref(h)), "matrix_create_csr")
        self.h = h

    def update_values(self, vals):
        v = np.ascontiguousarray(vals, dtype=np.float64)
        self.ctx.check(lib().ab2_matrix_update_values(self.ctx.h, self.h, _dp(v)), "update_values")
        self.vals = v

    @property
    def info(self) -> MatrixInfo:
        i = MatrixInfo()
        self.ctx.check(lib().ab2_matrix_get_info(self.h, C.byref(i)))
        return i

    def close(self):
        if self.h:
            lib().ab2_matrix_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Vector:
    def __init__(self, ctx: Context, n: int, handle=None):
        self.ctx = ctx
        self.n = n
        if handle is not None:  # created elsewhere (ab2_dist_vector_create)
            self.h = handle
            return
        h = _P()
        ctx.check(lib().ab2_vector_create(ctx.h, n, C.byref(h)), "vector_create")
        self.h = h

    def upload(self, a):
        a = np.ascontiguousarray(a, dtype=np.float64)
        assert a.size == self.n
        self.ctx.check(lib().ab2_vector_upload(self.ctx.h, self.h, _dp(a)), "upload")

    def download(self, out: np.ndarray | None = None) -> np.ndarray:
        """The vector's values; into `out` (contiguous float64, e.g. pinned memory) when given."""
        if out is None:
            out = np.empty(self.n, dtype=np.float64)
        assert out.dtype == np.float64 and out.size == self.n and out.flags.c_contiguous
        self.ctx.check(lib().ab2_vector_download(self.ctx.h, self.h, _dp(out)), "download")
        return out

    @property
    def device_ptr(self) -> int:
        p = _P()
        self.ctx.check(lib().ab2_vector_device_ptr(self.h, C.byref(p)))
        return p.value or 0

    def close(self):
        if self.h:
            lib().ab2_vector_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Precond:
    def __init__(self, ctx: Context, A: Matrix, kind: str = "diag", poly_factor: float = 0.0, poly_order: int = 3,
                 poly_factor_max_iter: int = 10, ilu_schedule: str = "auto", cheb_saad: bool = False,
                 cheb_lanczos: bool = False, filu_factor_iter: int = 0, filu_solver_iter: int = 3,
                 filu_tol: float = 0.0):
        self.ctx, self.A = ctx, A
        o = PrecondOptions(PRECOND[kind], poly_factor, poly_order, poly_factor_max_iter, ILU_SCHEDULE[ilu_schedule],
                           int(cheb_saad), int(cheb_lanczos), filu_factor_iter, filu_solver_iter, filu_tol)
        h = _P()
        ctx.check(lib().ab2_precond_create(ctx.h, A.h, C.byref(o), C.byref(h)), "precond_create")
        self.h = h

    def apply(self, x: Vector, y: Vector):
        self.ctx.check(lib().ab2_precond_apply(self.ctx.h, self.h, x.h, y.h), "precond_apply")

    @property
    def info(self) -> PrecondInfo:
        i = PrecondInfo()
        self.ctx.check(lib().ab2_precond_get_info(self.h, C.byref(i)))
        return i

    def ilu0_values(self) -> np.ndarray:
        out = np.empty(self.A.cols.size, dtype=np.float64)
        self.ctx.check(lib().ab2_precond_ilu0_values(self.ctx.h, self.h, _dp(out)), "ilu0_values")
        return out

    def close(self):
        if self.h:
            lib().ab2_precond_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


@dataclass
class SolveResult:
    succeeded: bool
    iterations: int
    error: int
    breakdown: str | None
    residual: float
    true_residual: float
    nrm2_b: float
    setup_ms: float
    solve_ms: float


def solver_options(solver="cg", precond="diag", tol=1e-8, max_iter=1000, poly_factor=0.0, poly_order=3,
                   poly_factor_max_iter=10, spmv_variant=SPMV_AUTO, use_graph=True,
                   ilu_schedule="auto", cheb_saad=False, cheb_lanczos=False, filu_factor_iter=0,
                   filu_solver_iter=3, filu_tol=0.0) -> SolverOptions:
    o = SolverOptions()
    lib().ab2_solver_options_default(C.byref(o))
    o.solver = SOLVER[solver]
    o.precond = PRECOND[precond]
    o.tol = tol
    o.max_iter = max_iter
    o.poly_factor = poly_factor
    o.poly_order = poly_order
    o.poly_factor_max_iter = poly_factor_max_iter
    o.spmv_variant = spmv_variant
    o.use_graph = 1 if use_graph else 0
    o.ilu_schedule = ILU_SCHEDULE[ilu_schedule]
    o.cheb_saad = int(cheb_saad)
    o.cheb_lanczos = int(cheb_lanczos)
    o.filu_factor_iter = filu_factor_iter
    o.filu_solver_iter = filu_solver_iter
    o.filu_tol = filu_tol
    return o


class Solver:
    """ab2_solver: preconditioner set-up at construction, device-resident loop in solve()."""

    def __init__(self, ctx: Context, A: Matrix, **opts):
        self.ctx, self.A = ctx, A
        self.opts = solver_options(**opts)
        h = _P()
        ctx.check(lib().ab2_solver_create(ctx.h, A.h, C.byref(self.opts), C.byref(h)), "solver_create")
        self.h = h

    def solve(self, b: Vector, x: Vector) -> SolveResult:
        st = Status()
        self.ctx.check(lib().ab2_solver_solve(self.h, b.h, x.h, C.byref(st)), "solve")
        return SolveResult(bool(st.succeeded), st.iterations, st.error, BREAKDOWN.get(st.breakdown), st.residual,
                           st.true_residual, st.nrm2_b, st.setup_ms, st.solve_ms)

    def history(self) -> np.ndarray:
        n = C.c_int()
        lib().ab2_solver_history(self.h, None, 0, C.byref(n))
        out = np.empty(max(n.value, 0), dtype=np.float64)
        if n.value:
            self.ctx.check(lib().ab2_solver_history(self.h, _dp(out), n.value, C.byref(n)), "history")
        return out

    def close(self):
        if self.h:
            lib().ab2_solver_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass



# ---------------------------------------------------------------------------- row-block distribution
class Comm:
    """One rank of an ab2_comm (include/ab2_dist.h).  Collective calls must be
    made by every rank in the same order; with a local group each rank is
    driven by its own thread (ctypes releases the GIL during the calls)."""

    def __init__(self, ctx: Context, handle):
        self.ctx, self.h = ctx, handle

    @staticmethod
    def local_group(ctxs: list[Context], timeout_s: float = 120.0) -> list["Comm"]:
        k = len(ctxs)
        arr = (_P * k)(*[c.h for c in ctxs])
        out = (_P * k)()
        ctxs[0].check(lib().ab2_comm_local_group(arr, k, timeout_s, out), "comm_local_group")
        return [Comm(c, _P(out[i])) for i, c in enumerate(ctxs)]

    @staticmethod
    def nccl_unique_id() -> bytes:
        buf = (C.c_ubyte * COMM_ID_BYTES)()
        rc = lib().ab2_comm_nccl_unique_id(buf)
        if rc != AB2_OK:
            raise AB2Error(rc, "comm_nccl_unique_id")
        return bytes(buf)

    @staticmethod
    def nccl(ctx: Context, uid: bytes, rank: int, size: int) -> "Comm":
        buf = (C.c_ubyte * COMM_ID_BYTES).from_buffer_copy(uid)
        h = _P()
        ctx.check(lib().ab2_comm_nccl_create(ctx.h, buf, rank, size, C.byref(h)), "comm_nccl_create")
        return Comm(ctx, h)

    @property
    def rank(self) -> int:
        r = C.c_int()
        lib().ab2_comm_rank(self.h, C.byref(r))
        return r.value

    @property
    def size(self) -> int:
        r = C.c_int()
        lib().ab2_comm_size(self.h, C.byref(r))
        return r.value

    def dot(self, x: Vector, y: Vector) -> float:
        r = C.c_double()
        self.ctx.check(lib().ab2_dist_dot(self.ctx.h, self.h, x.h, y.h, C.byref(r)), "dist_dot")
        return r.value

    def norm1(self, x: Vector) -> float:
        r = C.c_double()
        self.ctx.check(lib().ab2_dist_norm1(self.ctx.h, self.h, x.h, C.byref(r)), "dist_norm1")
        return r.value

    def norm2(self, x: Vector) -> float:
        r = C.c_double()
        self.ctx.check(lib().ab2_dist_norm2(self.ctx.h, self.h, x.h, C.byref(r)), "dist_norm2")
        return r.value

    def close(self):
        if self.h:
            lib().ab2_comm_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class DistMatrix:
    """This rank's rows of a row-block distributed matrix (ab2_dist_matrix);
    cols in global numbering.  Creation is collective."""

    def __init__(self, ctx: Context, comm: Comm, offsets, row_ptr, cols, vals, formats: int = FMT_CSR | FMT_ELL):
        self.ctx, self.comm = ctx, comm
        self.offsets = np.ascontiguousarray(offsets, dtype=np.int32)
        rp = np.ascontiguousarray(row_ptr, dtype=np.int32)
        ci = np.ascontiguousarray(cols, dtype=np.int32)
        v = np.ascontiguousarray(vals, dtype=np.float64)
        h = _P()
        ctx.check(lib().ab2_dist_matrix_create(ctx.h, comm.h, _ip(self.offsets), _ip(rp), _ip(ci), _dp(v), formats,
                                               C.byref(h)), "dist_matrix_create")
        self.h = h
        self.n = int(self.offsets[comm.rank + 1] - self.offsets[comm.rank])

    @classmethod
    def from_global(cls, ctx: Context, comm: Comm, offsets, row_ptr, cols, vals, formats: int = FMT_CSR | FMT_ELL):
        """This rank's block of a global CSR matrix."""
        r = comm.rank
        a, b = int(offsets[r]), int(offsets[r + 1])
        rp = np.asarray(row_ptr)
        lo, hi = int(rp[a]), int(rp[b])
        return cls(ctx, comm, offsets, rp[a:b + 1] - lo, np.asarray(cols)[lo:hi], np.asarray(vals)[lo:hi], formats)

    @property
    def info(self) -> DistInfo:
        i = DistInfo()
        self.ctx.check(lib().ab2_dist_matrix_get_info(self.h, C.byref(i)))
        return i

    def layout(self) -> dict:
        i = self.info
        nnz = i.local_nnz + i.ghost_nnz
        out = dict(row_ptr=np.empty(i.local_rows + 1, np.int32), cols=np.empty(nnz, np.int32),
                   vals=np.empty(nnz, np.float64), local_row_size=np.empty(i.local_rows, np.int32),
                   ghost_uids=np.empty(i.ghost_rows, np.int32), interface_rows=np.empty(i.interface_rows, np.int32))
        self.ctx.check(lib().ab2_dist_matrix_layout(self.h, _ip(out["row_ptr"]), _ip(out["cols"]), _dp(out["vals"]),
                                                    _ip(out["local_row_size"]), _ip(out["ghost_uids"]),
                                                    _ip(out["interface_rows"])))
        return out

    def plan(self) -> dict:
        i = self.info
        out = dict(recv_ranks=np.empty(i.recv_neighbours, np.int32), recv_offsets=np.empty(i.recv_neighbours + 1, np.int32),
                   send_ranks=np.empty(i.send_neighbours, np.int32), send_offsets=np.empty(i.send_neighbours + 1, np.int32),
                   send_ids=np.empty(i.send_count, np.int32))
        self.ctx.check(lib().ab2_dist_matrix_plan(self.h, _ip(out["recv_ranks"]), _ip(out["recv_offsets"]),
                                                  _ip(out["send_ranks"]), _ip(out["send_offsets"]), _ip(out["send_ids"])))
        return out

    def vector(self, values=None) -> Vector:
        """A vector of this rank's rows with room for the ghost values."""
        h = _P()
        self.ctx.check(lib().ab2_dist_vector_create(self.ctx.h, self.h, C.byref(h)), "dist_vector_create")
        v = Vector(self.ctx, self.n, handle=h)
        if values is not None:
            v.upload(values)
        return v

    def mult(self, x: Vector, y: Vector):
        self.ctx.check(lib().ab2_dist_mult(self.ctx.h, self.h, x.h, y.h), "dist_mult")

    def close(self):
        if self.h:
            lib().ab2_dist_matrix_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class DistPrecond(Precond):
    """NONE, DIAG or block-Jacobi ILU0 over this rank's rows (ab2_dist_precond_create)."""

    def __init__(self, ctx: Context, A: DistMatrix, kind: str = "ilu0", ilu_schedule: str = "auto"):
        self.ctx, self.A = ctx, A
        o = PrecondOptions(PRECOND[kind], 0.0, 3, 10, ILU_SCHEDULE[ilu_schedule], 0, 0, 0, 3, 0.0)
        h = _P()
        ctx.check(lib().ab2_dist_precond_create(ctx.h, A.h, C.byref(o), C.byref(h)), "dist_precond_create")
        self.h = h

    def ilu0_values(self) -> np.ndarray:
        out = np.empty(self.A.info.local_nnz, dtype=np.float64)
        self.ctx.check(lib().ab2_precond_ilu0_values(self.ctx.h, self.h, _dp(out)), "ilu0_values")
        return out


class DistSolver:
    """ab2_dist_solver: CG or BiCGStab on the distributed algebra, device-resident; solve() is collective."""

    def __init__(self, ctx: Context, comm: Comm, A: DistMatrix, **opts):
        self.ctx, self.comm, self.A = ctx, comm, A
        self.opts = solver_options(**opts)
        h = _P()
        ctx.check(lib().ab2_dist_solver_create(ctx.h, comm.h, A.h, C.byref(self.opts), C.byref(h)),
                  "dist_solver_create")
        self.h = h

    def solve(self, b: Vector, x: Vector) -> SolveResult:
        st = Status()
        self.ctx.check(lib().ab2_dist_solver_solve(self.h, b.h, x.h, C.byref(st)), "dist_solve")
        return SolveResult(bool(st.succeeded), st.iterations, st.error, BREAKDOWN.get(st.breakdown), st.residual,
                           st.true_residual, st.nrm2_b, st.setup_ms, st.solve_ms)

    def history(self) -> np.ndarray:
        n = C.c_int()
        lib().ab2_dist_solver_history(self.h, None, 0, C.byref(n))
        out = np.empty(max(n.value, 0), dtype=np.float64)
        if n.value:
            self.ctx.check(lib().ab2_dist_solver_history(self.h, _dp(out), n.value, C.byref(n)), "history")
        return out

    def close(self):
        if self.h:
            lib().ab2_dist_solver_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def row_offsets(n: int, nranks: int, align: int = 1) -> np.ndarray:
    """Contiguous row blocks of nearly equal size (multiples of align rows,
    e.g. a grid plane, except the last block)."""
    units = -(-n // align)
    cuts = [min(n, (units * r // nranks) * align) for r in range(nranks)] + [n]
    return np.asarray(cuts, dtype=np.int32)


@dataclass
class MixedResult:
    succeeded: bool
    outer_iterations: int
    inner_iterations: int
    error: int
    true_residual: float
    setup_ms: float
    solve_ms: float
    jacobi_scaled: bool = False


def mixed_options(solver="cg", precond="diag", tol=1e-8, max_outer=20, inner_tol=1e-4, inner_max_iter=1000,
                  poly_factor=0.0, poly_order=3, poly_factor_max_iter=20, cheb_saad=False, cheb_lanczos=False,
                  ilu_schedule="auto", spmv_variant=SPMV_AUTO, use_graph=True, filu_factor_iter=0,
                  filu_solver_iter=3, filu_tol=0.0, jacobi_form="auto") -> MixedOptions:
    o = MixedOptions()
    lib().ab2_mixed_options_default(C.byref(o))
    o.solver = SOLVER[solver]
    o.precond = PRECOND[precond]
    o.tol = tol
    o.max_outer = max_outer
    o.inner_tol = inner_tol
    o.inner_max_iter = inner_max_iter
    o.poly_factor = poly_factor
    o.poly_order = poly_order
    o.poly_factor_max_iter = poly_factor_max_iter
    o.cheb_saad = int(cheb_saad)
    o.cheb_lanczos = int(cheb_lanczos)
    o.ilu_schedule = ILU_SCHEDULE[ilu_schedule]
    o.spmv_variant = spmv_variant
    o.use_graph = 1 if use_graph else 0
    o.filu_factor_iter = filu_factor_iter
    o.filu_solver_iter = filu_solver_iter
    o.filu_tol = filu_tol
    o.jacobi_form = MIXED_JACOBI[jacobi_form]
    return o


class Mixed:
    """ab2_mixed: FP32 CG/BiCGStab inside FP64 iterative refinement (the matrix
    needs FMT_F32)."""

    def __init__(self, ctx: Context, A: Matrix, **opts):
        self.ctx, self.A = ctx, A
        self.opts = mixed_options(**opts)
        h = _P()
        ctx.check(lib().ab2_mixed_create(ctx.h, A.h, C.byref(self.opts), C.byref(h)), "mixed_create")
        self.h = h

    def solve(self, b: Vector, x: Vector) -> MixedResult:
        st = MixedStatus()
        self.ctx.check(lib().ab2_mixed_solve(self.h, b.h, x.h, C.byref(st)), "mixed_solve")
        return MixedResult(bool(st.succeeded), st.outer_iterations, st.inner_iterations, st.error,
                           st.true_residual, st.setup_ms, st.solve_ms, bool(st.jacobi_scaled))

    def history(self) -> np.ndarray:
        n = C.c_int()
        lib().ab2_mixed_history(self.h, None, 0, C.byref(n))
        out = np.empty(max(n.value, 0), dtype=np.float64)
        if n.value:
            self.ctx.check(lib().ab2_mixed_history(self.h, _dp(out), n.value, C.byref(n)), "mixed_history")
        return out

    def close(self):
        if self.h:
            lib().ab2_mixed_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


@dataclass
class BatchResult:
    systems_converged: int
    max_outer: int
    inner_total: int
    inner_max: int
    max_residual: float
    solve_ms: float


class Batch:
    """ab2_batch: independent systems (diagonal blocks of A, rows
    sys_offsets[s]..sys_offsets[s+1]-1) solved in one persistent launch; A
    needs FMT_F32.  cluster_size / threads / spmv_variant / ell_slice /
    lanes_per_row = 0 / 0 / SPMV_AUTO / 0 / 0 let the autotuner pick."""

    def __init__(self, ctx: Context, A: Matrix, sys_offsets, tol=1e-8, max_outer=20, inner_tol=1e-4,
                 inner_max_iter=5000, spmv_variant=SPMV_AUTO, cluster_size=0, threads=0, tune_iters=8, ell_slice=0,
                 lanes_per_row=0):
        self.ctx, self.A = ctx, A
        self.offsets = np.ascontiguousarray(sys_offsets, dtype=np.int32)
        self.nsys = self.offsets.size - 1
        o = BatchOptions()
        lib().ab2_batch_options_default(C.byref(o))
        o.tol, o.max_outer, o.inner_tol, o.inner_max_iter = tol, max_outer, inner_tol, inner_max_iter
        o.spmv_variant, o.cluster_size, o.threads, o.tune_iters = spmv_variant, cluster_size, threads, tune_iters
        o.ell_slice, o.lanes_per_row = ell_slice, lanes_per_row
        h = _P()
        ctx.check(lib().ab2_batch_create(ctx.h, A.h, self.nsys, _ip(self.offsets), C.byref(o), C.byref(h)),
                  "batch_create")
        self.h = h

    def solve(self, b: Vector, x: Vector) -> BatchResult:
        st = BatchStatus()
        self.ctx.check(lib().ab2_batch_solve(self.h, b.h, x.h, C.byref(st)), "batch_solve")
        return BatchResult(st.systems_converged, st.max_outer, st.inner_total, st.inner_max, st.max_residual,
                           st.solve_ms)

    def results(self):
        conv = np.empty(self.nsys, dtype=np.int32)
        outer = np.empty(self.nsys, dtype=np.int32)
        inner = np.empty(self.nsys, dtype=np.int32)
        res = np.empty(self.nsys)
        self.ctx.check(lib().ab2_batch_results(self.h, _ip(conv), _ip(outer), _ip(inner), _dp(res)), "batch_results")
        return conv.astype(bool), outer, inner, res

    @property
    def info(self) -> BatchInfo:
        i = BatchInfo()
        self.ctx.check(lib().ab2_batch_get_info(self.h, C.byref(i)), "batch_info")
        return i

    def trials(self) -> list[tuple[int, int, int, float, int, int]]:
        """(spmv_variant, cluster_size, threads, ms, ell_slice, lanes_per_row) per autotuning trial."""
        n = self.info.trials
        arr = (BatchTrial * max(n, 1))()
        self.ctx.check(lib().ab2_batch_trials(self.h, arr, n), "batch_trials")
        return [(t.spmv_variant, t.cluster_size, t.threads, t.ms, t.ell_slice, t.lanes_per_row) for t in arr[:n]]

    def close(self):
        if self.h:
            lib().ab2_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _fp32(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_float))


class Gnn:
    """ab2_gnn: the learned preconditioner (network on the matrix graph),
    trained on the GPU by libab2's own forward/backward kernels."""

    def __init__(self, ctx: Context, params=None, seed: int = 0):
        self.ctx = ctx
        h = _P()
        p = None if params is None else np.ascontiguousarray(params, dtype=np.float32)
        if p is not None and p.size != self.param_count():
            raise ValueError(f"expected {self.param_count()} parameters, got {p.size}")
        ctx.check(lib().ab2_gnn_create(ctx.h, None if p is None else _fp32(p), seed, C.byref(h)), "gnn_create")
        self.h = h
        self.A = None

    @staticmethod
    def param_count() -> int:
        return lib().ab2_gnn_param_count()

    @property
    def params(self) -> np.ndarray:
        out = np.empty(self.param_count(), dtype=np.float32)
        self.ctx.check(lib().ab2_gnn_get_params(self.h, _fp32(out)), "gnn_get_params")
        return out

    @params.setter
    def params(self, p):
        p = np.ascontiguousarray(p, dtype=np.float32)
        self.ctx.check(lib().ab2_gnn_set_params(self.h, _fp32(p)), "gnn_set_params")

    def set_layer(self, layer: str):
        """'auto', 'gather' or 'grid' (takes effect at the next bind)."""
        self.ctx.check(lib().ab2_gnn_set_layer(self.h, GNN_LAYER[layer]), "gnn_set_layer")

    @property
    def layer(self) -> str:
        v = C.c_int()
        self.ctx.check(lib().ab2_gnn_get_layer(self.h, C.byref(v)), "gnn_get_layer")
        return next(k for k, c in GNN_LAYER.items() if c == v.value)

    def bind(self, A: Matrix):
        self.ctx.check(lib().ab2_gnn_bind(self.h, A.h), "gnn_bind")
        self.A = A

    def apply(self, r: Vector, z: Vector):
        self.ctx.check(lib().ab2_gnn_apply(self.h, r.h, z.h), "gnn_apply")

    def loss_grad(self, r: Vector, e: Vector):
        L = C.c_double()
        g = np.empty(self.param_count(), dtype=np.float32)
        self.ctx.check(lib().ab2_gnn_loss_grad(self.h, r.h, e.h, C.byref(L), _fp32(g)), "gnn_loss_grad")
        return L.value, g

    def train_step(self, r: Vector, e: Vector, lr: float = 1e-3) -> float:
        L = C.c_double()
        self.ctx.check(lib().ab2_gnn_train_step(self.h, r.h, e.h, lr, C.byref(L)), "gnn_train_step")
        return L.value

    def close(self):
        if self.h:
            lib().ab2_gnn_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


@dataclass
class FcgResult:
    succeeded: bool
    iterations: int
    gnn_steps: int
    fallback_steps: int
    switched_at: int
    error: int
    true_residual: float
    solve_ms: float


def fcg_solve(ctx: Context, A: Matrix, b: Vector, x: Vector, gnn: Gnn | None = None, fallback: "Precond | None" = None,
              tol: float = 1e-8, max_iter: int = 5000, fallback_ratio: float = 1.0,
              truncation: int | None = None, fallback_mode: str | None = None) -> FcgResult:
    """Flexible CG (truncated A-orthogonalisation over `truncation` directions)
    with the learned preconditioner, the fallback (ILU0) taking over from the
    first network step that reduces ||r|| by less than fallback_ratio."""
    o = FcgOptions()
    lib().ab2_fcg_options_default(C.byref(o))
    o.tol, o.max_iter, o.fallback_ratio = tol, max_iter, fallback_ratio
    if truncation is not None:
        o.truncation = truncation
    if fallback_mode is not None:
        o.fallback_mode = FCG_FALLBACK[fallback_mode]
    st = FcgStatus()
    ctx.check(lib().ab2_fcg_solve(ctx.h, A.h, gnn.h if gnn else None, fallback.h if fallback else None, b.h, x.h,
                                  C.byref(o), C.byref(st)), "fcg_solve")
    return FcgResult(bool(st.succeeded), st.iterations, st.gnn_steps, st.fallback_steps, st.switched_at, st.error,
                     st.true_residual, st.solve_ms)


# ---------------------------------------------------------------------------- problems
@dataclass
class CsrProblem:
    n: int
    row_ptr: np.ndarray
    cols: np.ndarray
    vals: np.ndarray
    x_true: np.ndarray
    b: np.ndarray
    log10_k: np.ndarray | None
    shape: tuple

    @property
    def nnz(self) -> int:
        return int(self.row_ptr[-1])


def _take(p) -> CsrProblem:
    P = p.contents
    n, nnz = P.n, P.nnz

    def arr(ptr, count, dt):
        return np.ctypeslib.as_array(ptr, shape=(count,)).astype(dt, copy=True)

    out = CsrProblem(n, arr(P.row_ptr, n + 1, np.int32), arr(P.cols, nnz, np.int32), arr(P.vals, nnz, np.float64),
                     arr(P.x_true, n, np.float64) if bool(P.x_true) else None, arr(P.b, n, np.float64),
                     arr(P.log10_k, n, np.float64) if bool(P.log10_k) else None, (P.nx, P.ny, P.nz))
    lib().ab2_problem_destroy(p)
    return out


def read_matrix_market(path, rhs=None) -> CsrProblem:
    """A MatrixMarket system as Alien's reader loads it (see
    include/ab2_problems.h); b = 1 without an rhs file; x_true is None."""
    p = C.POINTER(Problem)()
    rc = lib().ab2_problem_read_matrix_market(str(path).encode(), None if rhs is None else str(rhs).encode(),
                                              C.byref(p))
    if rc:
        raise AB2Error(rc, lib().ab2_matrix_market_error().decode())
    return _take(p)


def write_matrix_market(P: CsrProblem, path, rhs=None) -> None:
    """Writes P's matrix ("coordinate real general") and, with rhs, its b."""
    keep = [np.ascontiguousarray(P.row_ptr, np.int32), np.ascontiguousarray(P.cols, np.int32),
            np.ascontiguousarray(P.vals, np.float64), np.ascontiguousarray(P.b, np.float64)]
    pr = Problem()
    pr.n, pr.nnz, pr.nx, pr.ny, pr.nz = P.n, P.nnz, P.n, 1, 1
    pr.row_ptr = keep[0].ctypes.data_as(_IP)
    pr.cols = keep[1].ctypes.data_as(_IP)
    pr.vals = keep[2].ctypes.data_as(_DP)
    pr.b = keep[3].ctypes.data_as(_DP)
    rc = lib().ab2_problem_write_matrix_market(C.byref(pr), str(path).encode(),
                                               None if rhs is None else str(rhs).encode())
    if rc:
        raise AB2Error(rc, lib().ab2_matrix_market_error().decode())


def poisson(nx, ny=None, nz=None, seed=0) -> CsrProblem:
    ny = nx if ny is None else ny
    nz = nx if nz is None else nz
    p = C.POINTER(Problem)()
    rc = lib().ab2_problem_poisson(nx, ny, nz, seed, C.byref(p))
    if rc:
        raise AB2Error(rc, "ab2_problem_poisson")
    return _take(p)


def diffusion(nx, ny=None, nz=None, sigma=1.0, smooth=4.0, seed=0) -> CsrProblem:
    ny = nx if ny is None else ny
    nz = nx if nz is None else nz
    p = C.POINTER(Problem)()
    rc = lib().ab2_problem_diffusion(nx, ny, nz, sigma, smooth, seed, C.byref(p))
    if rc:
        raise AB2Error(rc, "ab2_problem_diffusion")
    return _take(p)


def convdiff(nx, ny=None, nz=None, peclet=10.0, modes=8, seed=0) -> CsrProblem:
    ny = nx if ny is None else ny
    nz = nx if nz is None else nz
    p = C.POINTER(Problem)()
    rc = lib().ab2_problem_convdiff(nx, ny, nz, peclet, modes, seed, C.byref(p))
    if rc:
        raise AB2Error(rc, "ab2_problem_convdiff")
    return _take(p)


@dataclass
class BatchProblem:
    """Independent systems stacked as one block-diagonal CSR matrix."""
    problem: CsrProblem
    sys_offsets: np.ndarray
    dims: list  # (nx, ny, nz) of each system

    @property
    def nsys(self) -> int:
        return self.sys_offsets.size - 1


def batch_problem(nsys=512, min_rows=2000, max_rows=200000, seed=0, sigma=1.0, smooth=2.0) -> BatchProblem:
    """nsys heterogeneous-diffusion systems (log10 k ~ smoothed N(0, sigma^2)),
    each 2-D 5-point or 3-D 7-point by a seeded coin, row counts log-uniform in
    [min_rows, max_rows] (grid side round(n^(1/d))), seed seed*100003 + s for
    system s, stacked as the diagonal blocks of one CSR matrix."""
    lib()
    parts, dims = [], []
    for s in range(nsys):
        u0 = 0.5 * (lib().ab2_rng_uniform(seed, 1000 + s, 0) + 1.0)  # U[0, 1)
        u1 = 0.5 * (lib().ab2_rng_uniform(seed, 1000 + s, 1) + 1.0)
        n = float(np.exp(np.log(min_rows) + u0 * (np.log(max_rows) - np.log(min_rows))))
        if u1 < 0.5:
            side = max(2, int(round(n ** 0.5)))
            dim = (side, side, 1)
        else:
            side = max(2, int(round(n ** (1 / 3))))
            dim = (side, side, side)
        P = diffusion(*dim, sigma=sigma, smooth=smooth, seed=seed * 100003 + s)
        parts.append(P)
        dims.append(dim)
    offs = np.zeros(nsys + 1, dtype=np.int64)
    for s, P in enumerate(parts):
        offs[s + 1] = offs[s] + P.n
    nnz = sum(P.nnz for P in parts)
    rp = np.empty(int(offs[-1]) + 1, dtype=np.int64)
    ci = np.empty(nnz, dtype=np.int32)
    vals = np.empty(nnz)
    xt = np.empty(int(offs[-1]))
    b = np.empty(int(offs[-1]))
    e = 0
    rp[0] = 0
    for s, P in enumerate(parts):
        o = int(offs[s])
        rp[o + 1:o + P.n + 1] = P.row_ptr[1:].astype(np.int64) + e
        ci[e:e + P.nnz] = P.cols + o
        vals[e:e + P.nnz] = P.vals
        xt[o:o + P.n] = P.x_true
        b[o:o + P.n] = P.b
        e += P.nnz
    assert rp[-1] < 2**31
    prob = CsrProblem(int(offs[-1]), rp.astype(np.int32), ci, vals, xt, b, None, (int(offs[-1]), 1, 1))
    return BatchProblem(prob, offs.astype(np.int32), dims)
