"""Test inputs: seeded generator systems plus hand-made ragged CSR matrices."""
from __future__ import annotations

import functools

import numpy as np

from alien_b200 import abi


@functools.lru_cache(maxsize=None)
def get(name: str) -> abi.CsrProblem:
    if name == "poisson16":
        return abi.poisson(16, 16, 16, seed=0)
    if name == "poisson32":  # the 32^3 constant-coefficient system, seed 0
        return abi.poisson(32, 32, 32, seed=0)
    if name == "poisson2d_23x17":
        return abi.poisson(23, 17, 1, seed=3)
    if name == "diffusion12":
        return abi.diffusion(12, 12, 12, sigma=1.0, smooth=2.0, seed=1)
    if name == "diffusion24":
        return abi.diffusion(24, 24, 24, sigma=1.0, smooth=4.0, seed=5)
    if name == "diffusion64":
        return abi.diffusion(64, 64, 64, sigma=1.0, smooth=4.0, seed=0)
    if name == "diffusion_10x11x12":  # nx not a multiple of 4
        return abi.diffusion(10, 11, 12, sigma=1.0, smooth=2.0, seed=8)
    if name == "diffusion_20x6x9":
        return abi.diffusion(20, 6, 9, sigma=1.0, smooth=2.0, seed=9)
    if name == "diffusion_80x72x64":  # more rows than one sweep of the largest reduction grid
        return abi.diffusion(80, 72, 64, sigma=1.0, smooth=4.0, seed=10)
    if name == "diffusion2d_31x9":
        return abi.diffusion(31, 9, 1, sigma=1.5, smooth=3.0, seed=7)
    if name == "convdiff_10x11x12":
        return abi.convdiff(10, 11, 12, peclet=10.0, modes=8, seed=2)
    if name == "convdiff16":
        return abi.convdiff(16, 16, 16, peclet=10.0, modes=8, seed=4)
    if name == "ragged":
        return ragged(1000, seed=11)
    if name == "longrow":
        return long_row_matrix()
    if name.startswith("wide"):  # wide<mean>: rows of mean/4 .. 7 mean/4 entries
        return wide_rows(3001, int(name[4:]), seed=17)
    raise KeyError(name)


def ragged(n: int, seed: int) -> abi.CsrProblem:
    """Diagonally dominant nonsymmetric CSR with uneven rows (0..40 off-diagonals,
    some rows diagonal-only), n not a multiple of 32."""
    rng = np.random.default_rng(seed)
    rows = []
    for i in range(n):
        k = 0 if i % 17 == 0 else int(rng.integers(0, 41))
        cols = set(rng.choice(n, size=min(k, n - 1), replace=False).tolist()) - {i}
        rows.append(sorted(cols | {i}))
    row_ptr = np.zeros(n + 1, dtype=np.int32)
    cols, vals = [], []
    for i, cs in enumerate(rows):
        off = rng.uniform(-1, 1, size=len(cs))
        d = float(np.sum(np.abs(off))) + 1.0
        for c, v in zip(cs, off):
            cols.append(c)
            vals.append(d if c == i else v)
        row_ptr[i + 1] = row_ptr[i] + len(cs)
    cols = np.asarray(cols, dtype=np.int32)
    vals = np.asarray(vals, dtype=np.float64)
    x_true = rng.uniform(-1, 1, size=n)
    from oracle import oracle as O

    b = O.spmv(row_ptr, cols, vals, x_true)
    return abi.CsrProblem(n, row_ptr, cols, vals, x_true, b, None, (n, 1, 1))


def long_row_matrix(n: int = 4000, seed: int = 13) -> abi.CsrProblem:
    """A matrix whose middle row has every column (longer than any staging block)."""
    rng = np.random.default_rng(seed)
    row_ptr = [0]
    cols, vals = [], []
    for i in range(n):
        cs = list(range(n)) if i == n // 2 else sorted({i, (i + 1) % n, (i * 7 + 3) % n})
        for c in cs:
            cols.append(c)
            vals.append(float(len(cs) + 1) if c == i else float(rng.uniform(-1, 1)))
        row_ptr.append(len(cols))
    row_ptr = np.asarray(row_ptr, dtype=np.int32)
    cols = np.asarray(cols, dtype=np.int32)
    vals = np.asarray(vals)
    x_true = rng.uniform(-1, 1, size=n)
    from oracle import oracle as O

    return abi.CsrProblem(n, row_ptr, cols, vals, x_true, O.spmv(row_ptr, cols, vals, x_true), None, (n, 1, 1))


def wide_rows(n: int, mean: int, seed: int) -> abi.CsrProblem:
    """Rows of uniform random length in [mean/4, 7 mean/4] (at least 1), the
    diagonal plus columns spread at stride n / length, diagonally dominant."""
    rng = np.random.default_rng(seed)
    lens = np.maximum(1, rng.integers(mean // 4, 7 * mean // 4 + 1, n))
    row_ptr = np.zeros(n + 1, np.int64)
    np.cumsum(lens, out=row_ptr[1:])
    row = np.repeat(np.arange(n), lens)
    j = np.arange(row_ptr[-1]) - row_ptr[row]
    cols = (row + j * (n // lens[row])) % n
    order = np.argsort(row * n + cols, kind="stable")
    cols = cols[order].astype(np.int32)
    vals = rng.uniform(-1, 1, row_ptr[-1])
    vals[cols == row] = lens + 1.0
    row_ptr = row_ptr.astype(np.int32)
    x_true = rng.uniform(-1, 1, size=n)
    from oracle import oracle as O

    return abi.CsrProblem(n, row_ptr, cols, vals, x_true, O.spmv(row_ptr, cols, vals, x_true), None, (n, 1, 1))


def laplacian_1d(n: int = 10):
    """The 10-row (2, -1) Laplacian of Alien's TestMVExpr.cc:34-63."""
    row_ptr = [0]
    cols, vals = [], []
    for i in range(n):
        for c, v in ((i - 1, -1.0), (i, 2.0), (i + 1, -1.0)):
            if 0 <= c < n:
                cols.append(c)
                vals.append(v)
        row_ptr.append(len(cols))
    return np.asarray(row_ptr, np.int32), np.asarray(cols, np.int32), np.asarray(vals)
