"""The host-only build of the seeded input generators (oracle/_build/
libab2_inputs.so, used by the CPU reference timing so that it never loads the
CUDA library) makes the same systems as libab2, bit for bit (no GPU needed:
both libraries load on a CPU-only host)."""
import numpy as np
import pytest

from alien_b200 import abi
from oracle import oracle as O

CASES = [
    ("poisson", dict(nx=17, ny=9, nz=5, seed=3)),
    ("poisson", dict(nx=32, ny=32, nz=32, seed=0)),
    ("diffusion", dict(nx=33, ny=1, nz=1, sigma=1.0, smooth=4.0, seed=1)),
    ("diffusion", dict(nx=40, ny=37, nz=1, sigma=1.5, smooth=2.5, seed=7)),
    ("diffusion", dict(nx=48, ny=48, nz=48, sigma=1.0, smooth=4.0, seed=0)),
    ("convdiff", dict(nx=24, ny=20, nz=16, peclet=10.0, modes=8, seed=2)),
]


def _fields(P):
    return (P.n, P.nnz, tuple(P.shape), P.row_ptr, P.cols, P.vals, P.x_true, P.b, P.log10_k)


@pytest.mark.parametrize("kind,kw", CASES, ids=[f"{k}-{i}" for i, (k, _) in enumerate(CASES)])
def test_host_generator_is_libab2s(kind, kw):
    a = getattr(abi, kind)(**kw)
    b = getattr(O, f"problem_{kind}")(**kw)
    fa, fb = _fields(a), _fields(b)
    assert fa[:3] == fb[:3]
    for u, v in zip(fa[3:], fb[3:]):
        if u is None or v is None:
            assert u is None and v is None
            continue
        assert u.dtype == v.dtype and u.shape == v.shape
        assert u.tobytes() == v.tobytes()
