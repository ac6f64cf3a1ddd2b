"""libab2's C ABI surface and its host-side generators (no GPU needed)."""
import ctypes as C
import re
from pathlib import Path

import numpy as np
import pytest

from alien_b200 import abi
from oracle import oracle as O
from tests import problems

INCLUDE = Path(__file__).resolve().parents[1] / "include"


def declared_symbols():
    names = set()
    for h in INCLUDE.glob("*.h"):
        text = h.read_text()
        names |= set(re.findall(r"\b(ab2_[a-z0-9_]+)\s*\(", text))
    return names


def test_library_loads_and_exports_every_declared_symbol():
    L = abi.lib()
    names = declared_symbols()
    assert len(names) > 40
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing
    # and the Python binding types every one of them
    assert names == set(abi.SIGNATURES), names ^ set(abi.SIGNATURES)


def test_bad_arguments_are_rejected_without_a_device():
    L = abi.lib()
    assert L.ab2_context_create(0, None) == abi.AB2_ERR_BAD_ARG
    assert L.ab2_matrix_create_csr(None, 0, None, None, None, 0, None) == abi.AB2_ERR_BAD_ARG
    assert L.ab2_dot(None, None, None, None) == abi.AB2_ERR_BAD_ARG
    assert L.ab2_solver_solve(None, None, None, None) == abi.AB2_ERR_BAD_ARG
    assert L.ab2_problem_poisson(0, 1, 1, 0, None) == abi.AB2_ERR_BAD_ARG


def test_rng_streams_are_counter_based():
    L = abi.lib()
    a = [L.ab2_rng_uniform(7, 0, i) for i in range(1000)]
    assert all(-1.0 <= v < 1.0 for v in a)
    assert abs(np.mean(a)) < 0.1
    assert L.ab2_rng_u64(7, 0, 5) == L.ab2_rng_u64(7, 0, 5)
    assert L.ab2_rng_u64(7, 0, 5) != L.ab2_rng_u64(7, 1, 5)
    P = abi.poisson(8, 8, 8, seed=7)
    np.testing.assert_array_equal(P.x_true, np.array([L.ab2_rng_uniform(7, 0, i) for i in range(P.n)]))


@pytest.mark.parametrize("shape", [(32, 32, 32), (7, 5, 3), (23, 17, 1)])
def test_poisson_structure(shape):
    P = abi.poisson(*shape, seed=0)
    nx, ny, nz = shape
    d = 6.0 if nz > 1 else 4.0
    faces = (nx - 1) * ny * nz + nx * (ny - 1) * nz + (nx * ny * (nz - 1) if nz > 1 else 0)
    assert P.n == nx * ny * nz and P.nnz == P.n + 2 * faces
    if shape == (32, 32, 32):
        assert P.nnz == 223232
    for r in range(0, P.n, 97):
        cs = P.cols[P.row_ptr[r]:P.row_ptr[r + 1]]
        vs = P.vals[P.row_ptr[r]:P.row_ptr[r + 1]]
        assert np.all(np.diff(cs) > 0)
        assert vs[cs == r][0] == d and np.all(vs[cs != r] == -1.0)
    np.testing.assert_array_equal(P.b, O.spmv(P.row_ptr, P.cols, P.vals, P.x_true))


def _dense(P):
    A = np.zeros((P.n, P.n))
    for r in range(P.n):
        A[r, P.cols[P.row_ptr[r]:P.row_ptr[r + 1]]] = P.vals[P.row_ptr[r]:P.row_ptr[r + 1]]
    return A


def test_diffusion_is_spd_and_harmonic():
    P = problems.get("diffusion12")
    A = _dense(P)
    np.testing.assert_allclose(A, A.T, rtol=0, atol=0)
    assert np.all(np.linalg.eigvalsh(A) > 0)
    lg = P.log10_k
    assert abs(np.mean(lg)) < 1e-12 and abs(np.std(lg) - 1.0) < 1e-12
    k = 10.0 ** lg
    # face between cells 0 and 1 (x neighbours): harmonic mean
    t = 2 * k[0] * k[1] / (k[0] + k[1])
    row0 = dict(zip(P.cols[P.row_ptr[0]:P.row_ptr[1]], P.vals[P.row_ptr[0]:P.row_ptr[1]]))
    assert row0[1] == -t
    np.testing.assert_array_equal(P.b, O.spmv(P.row_ptr, P.cols, P.vals, P.x_true))


def test_diffusion_2d_is_five_point():
    P = problems.get("diffusion2d_31x9")
    assert P.shape == (31, 9, 1)
    assert max(np.diff(P.row_ptr)) == 5


def test_convdiff_is_an_m_matrix_with_peclet_bound():
    P = problems.get("convdiff16")
    A = _dense(P)
    off = A - np.diag(np.diag(A))
    assert np.all(off <= 0)
    assert np.all(np.diag(A) + off.sum(axis=1) >= -1e-9)  # weak diagonal dominance (div-free flow)
    conv = -off - (off != 0)  # the convective part of each off-diagonal
    assert conv.max() <= 10.0 + 1e-9 and conv.max() > 5.0
    assert not np.allclose(A, A.T)


def test_invalid_csr_rejected_on_host():
    L = abi.lib()
    rp = np.array([1, 2], dtype=np.int32)  # must start at 0
    ci = np.array([0], dtype=np.int32)
    v = np.array([1.0])
    h = C.c_void_p()
    # a NULL context is rejected before the profile is looked at
    assert L.ab2_matrix_create_csr(None, 1, rp.ctypes.data_as(C.POINTER(C.c_int)), ci.ctypes.data_as(
        C.POINTER(C.c_int)), v.ctypes.data_as(C.POINTER(C.c_double)), 1, C.byref(h)) == abi.AB2_ERR_BAD_ARG
