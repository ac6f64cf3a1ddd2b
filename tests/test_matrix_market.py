"""MatrixMarket input/output (host code in libab2), checked against the
reading rules of Alien's MatrixMarketReader.cc and against scipy's reader.

Rules (src/movesemantic/alien/move/impl/MatrixMarketReader.cc): only
"coordinate real" matrices; any symmetry other than "general" is mirrored with
the SAME value (so a skew-symmetric file comes out symmetric); duplicate
entries are summed in file order; '%' lines are comments.  Without a
right-hand-side file b = 1 (benchmark/src/alien/benchmark/MatrixMarketProblem.cpp)."""
import os
from pathlib import Path

import numpy as np
import pytest
import scipy.io
import scipy.sparse as sp

from alien_b200 import abi


def dense(P):
    A = np.zeros((P.n, P.n))
    for i in range(P.n):
        for k in range(P.row_ptr[i], P.row_ptr[i + 1]):
            A[i, P.cols[k]] += P.vals[k]
    return A


def test_round_trip_is_exact(tmp_path):
    P = abi.diffusion(7, 6, 5, sigma=1.5, smooth=2.0, seed=3)
    abi.write_matrix_market(P, tmp_path / "a.mtx", tmp_path / "b.mtx")
    Q = abi.read_matrix_market(tmp_path / "a.mtx", tmp_path / "b.mtx")
    assert Q.n == P.n and Q.x_true is None and Q.shape == (P.n, 1, 1)
    np.testing.assert_array_equal(Q.row_ptr, P.row_ptr)
    np.testing.assert_array_equal(Q.cols, P.cols)
    np.testing.assert_array_equal(Q.vals, P.vals)
    np.testing.assert_array_equal(Q.b, P.b)
    # scipy reads the same matrix and vector
    S = scipy.io.mmread(str(tmp_path / "a.mtx"))
    np.testing.assert_array_equal(sp.csr_matrix(S).toarray(), dense(Q))
    np.testing.assert_array_equal(np.asarray(scipy.io.mmread(str(tmp_path / "b.mtx"))).ravel(), Q.b)


def test_symmetric_duplicates_comments_and_default_rhs(tmp_path):
    f = tmp_path / "s.mtx"
    f.write_text("% leading comment line\n"
                 "%%MatrixMarket Matrix COORDINATE Real Symmetric\n"
                 "% comment\n\n"
                 "4 4 7\n"
                 "1 1 4.0\n"
                 "2 1 -1.0\n"
                 "% a comment between entries\n"
                 "2 2 4.0\n"
                 "3 2 -1.0\n"
                 "3 3 4.0\n"
                 "4 4 2.5\n"
                 "4 4 1.5\n")  # duplicate: summed
    P = abi.read_matrix_market(f)
    A = dense(P)
    expect = np.array([[4, -1, 0, 0], [-1, 4, -1, 0], [0, -1, 4, 0], [0, 0, 0, 4.0]])
    np.testing.assert_array_equal(A, expect)
    np.testing.assert_array_equal(P.b, np.ones(4))
    for i in range(P.n):  # columns ascending in every row
        assert np.all(np.diff(P.cols[P.row_ptr[i]:P.row_ptr[i + 1]]) > 0)
    # scipy wants the banner first and no comments among the entries (the reference reader does not)
    lines = f.read_text().splitlines()
    g = tmp_path / "s2.mtx"
    g.write_text("\n".join([lines[1]] + [ln for ln in lines[2:] if ln and not ln.startswith("%")]) + "\n")
    np.testing.assert_array_equal(sp.csr_matrix(scipy.io.mmread(str(g))).toarray(), expect)


def test_skew_symmetric_is_mirrored_with_the_same_sign(tmp_path):
    """The reference reader treats every non-general symmetry as symmetric."""
    f = tmp_path / "k.mtx"
    f.write_text("%%MatrixMarket matrix coordinate real skew-symmetric\n3 3 2\n2 1 0.5\n3 2 -2\n")
    A = dense(abi.read_matrix_market(f))
    np.testing.assert_array_equal(A, [[0, 0.5, 0], [0.5, 0, -2], [0, -2, 0]])


def test_duplicates_summed_in_file_order(tmp_path):
    f = tmp_path / "d.mtx"
    vals = [1e16, 1.0, -1e16, 1.0]  # order matters in floating point
    f.write_text("%%MatrixMarket matrix coordinate real general\n1 1 4\n" + "".join(f"1 1 {v!r}\n" for v in vals))
    acc = 0.0
    for v in vals:
        acc += v
    assert abi.read_matrix_market(f).vals[0] == acc


@pytest.mark.parametrize("text,rhs,msg", [
    ("%%MatrixMarket matrix coordinate integer general\n2 2 1\n1 1 3\n", None, "coordinate real"),
    ("%%MatrixMarket matrix coordinate pattern general\n2 2 1\n1 1\n", None, "coordinate real"),
    ("%%MatrixMarket matrix array real general\n2 2\n1\n2\n3\n4\n", None, "coordinate real"),
    ("%%MatrixMarket matrix coordinate real general\n2 3 1\n1 1 3\n", None, "square"),
    ("%%MatrixMarket matrix coordinate real general\n2 2 1\n3 1 3\n", None, "out of range"),
    ("%%MatrixMarket matrix coordinate real general\n2 2 3\n1 1 3\n", None, "ends"),
    ("no header\n2 2 1\n1 1 3\n", None, "header"),
    ("%%MatrixMarket matrix coordinate real general\n2 2 1\n1 1 3\n", "%%MatrixMarket matrix array real general\n3 1\n1\n2\n3\n", "size"),
    ("%%MatrixMarket matrix coordinate real general\n2 2 1\n1 1 3\n", "%%MatrixMarket matrix array real general\n2 2\n1\n2\n3\n4\n", "one vector"),
])
def test_bad_files_rejected(tmp_path, text, rhs, msg):
    f = tmp_path / "x.mtx"
    f.write_text(text)
    r = None
    if rhs is not None:
        r = tmp_path / "r.mtx"
        r.write_text(rhs)
    with pytest.raises(abi.AB2Error) as e:
        abi.read_matrix_market(f, r)
    assert e.value.code == abi.AB2_ERR_BAD_ARG and msg in str(e.value)


# The reference's own MatrixMarket fixtures, read where they lie in the
# reference checkout (ALIEN_REF_SRC, as oracle/Makefile: by default a checkout
# of arcaneframework/alien beside this repository; skipped when absent).
_REF_SRC = os.environ.get("ALIEN_REF_SRC") or str(Path(__file__).resolve().parents[2] / "reference" / "src" / "core")
REF_TESTS = Path(_REF_SRC).parent / "movesemantic" / "tests"


@pytest.mark.skipif(not (REF_TESTS / "simple.mtx").exists(), reason="reference checkout absent")
def test_reference_fixture_simple_mtx():
    """TestMatrixMarket.cc (movesemantic/tests): simple.mtx is 25 x 25 and
    simple_rhs.mtx holds i + 1 (floored) at row i, also per row block (the
    MatrixVector case reads the vector on the matrix's row distribution)."""
    P = abi.read_matrix_market(str(REF_TESTS / "simple.mtx"), str(REF_TESTS / "simple_rhs.mtx"))
    assert P.n == 25
    np.testing.assert_array_equal(np.floor(P.b), np.arange(1, 26))
    for off in ([0, 25], [0, 12, 25], [0, 7, 13, 25]):
        for a, b in zip(off[:-1], off[1:]):
            np.testing.assert_array_equal(np.floor(P.b[a:b]), np.arange(a, b) + 1)
    S = sp.csr_matrix(scipy.io.mmread(str(REF_TESTS / "simple.mtx")))
    S.sort_indices()
    np.testing.assert_array_equal(P.row_ptr, S.indptr)
    np.testing.assert_array_equal(P.cols, S.indices)
    np.testing.assert_array_equal(P.vals, S.data)
