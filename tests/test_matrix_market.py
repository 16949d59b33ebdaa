"""MatrixMarket reader and writer (tb_matrix_market_read / _write), on the host.

The reader is checked bit-exact against the reference's own
``Sparse::MatrixCSR::LoadFromMatrixMarket`` compiled from its headers (when the
reference checkout was available to build it) and against the oracle's
pure-Python restatement, on symmetric, general, pattern and integer files,
with comments, blank lines and multi-threaded parses; on repeated entries,
whose summation order the reference leaves to an unstable sort, bit-exact
against the restatement (file order) and to rounding against the reference.
Files the reference rejects are rejected here with a status.  The writer is
checked by its exact text and by bit-exact round trips.  One GPU test factors
and solves a matrix read from a file.
"""
from __future__ import annotations

import numpy as np
import pytest

import oracle
from tensors_b200 import matrices as M
from tensors_b200 import ordering as O
from tensors_b200.cholesky import CholeskyDecomposition, TBError
from tensors_b200.matrix_market import load_matrix_market, read_matrix_market, write_matrix_market

TB_ERR_IO, TB_ERR_FORMAT = -11, -12


def _same(a, b):
    assert a[0] == b[0] and a[1] == b[1]
    for x, y in zip(a[2:], b[2:]):
        assert x.dtype == y.dtype and np.array_equal(x, y)
    # values bit-exact (signed zeros included)
    assert np.array_equal(a[4].view(np.uint64), b[4].view(np.uint64))


def _checkers(path, threads=1):
    out = [oracle.mm_read_port(path)]
    if oracle.ref_available():
        out.append(oracle.ref_mm_read(path, threads))
    return out


def _write_triples(path, header, m, n, triples, fmt="{:.17g}"):
    with open(path, "w") as f:
        f.write(header + "\n% a comment line\n%\n")
        f.write(f"{m} {n} {len(triples)}\n")
        for t in triples:
            f.write(" ".join([str(t[0] + 1), str(t[1] + 1)] + [fmt.format(v) for v in t[2:]]) + "\n")


def _lower_triples(A: M.CSRMatrix):
    rows = np.repeat(np.arange(A.n), np.diff(A.outer))
    keep = A.inner <= rows
    return list(zip(rows[keep].tolist(), A.inner[keep].tolist(), A.values[keep].tolist()))


def test_symmetric_file_matches_reference(tmp_path):
    A = M.grid_laplacian_3d(9, 11, 1e-3)
    p = tmp_path / "sym.mtx"
    _write_triples(p, "%%MatrixMarket matrix coordinate real symmetric", A.n, A.n, _lower_triples(A))
    got = read_matrix_market(p)
    for want in _checkers(p):
        _same(got, want)
    # the full pattern of the generator, values included
    assert np.array_equal(got[2], A.outer) and np.array_equal(got[3], A.inner)
    assert np.array_equal(got[4], A.values)


def test_general_file_with_repeated_entries_matches_reference(tmp_path):
    rng = np.random.default_rng(7)
    m, n, k = 40, 35, 3000          # many (i, j) pairs repeat: summed in file order
    triples = [(int(i), int(j), float(v)) for i, j, v in
               zip(rng.integers(0, m, k), rng.integers(0, n, k), rng.standard_normal(k) * 10.0 ** rng.integers(-8, 8, k))]
    p = tmp_path / "gen.mtx"
    _write_triples(p, "%%MatrixMarket matrix coordinate real general", m, n, triples)
    got = read_matrix_market(p)
    assert got[0] == m and got[1] == n and int(got[2][-1]) < k
    _same(got, oracle.mm_read_port(p))
    if oracle.ref_available():
        # The reference orders a row's repeated columns with an unstable sort
        # (Ordering.hpp:24 through the utility module's Sort), so its summation
        # order is unspecified: the structure is exact, each sum agrees to the
        # rounding of c terms, |diff| <= c * eps * sum |a|.
        ref = oracle.ref_mm_read(p)
        assert ref[:2] == got[:2] and np.array_equal(ref[2], got[2]) and np.array_equal(ref[3], got[3])
        rows = np.repeat(np.arange(m), np.diff(got[2]))
        key = rows * n + got[3]
        ti = np.array([t[0] for t in triples]) * n + np.array([t[1] for t in triples])
        tv = np.abs(np.array([t[2] for t in triples]))
        count = np.array([np.sum(ti == q) for q in key])
        mag = np.array([tv[ti == q].sum() for q in key])
        assert np.all(np.abs(ref[4] - got[4]) <= count * np.finfo(float).eps * mag)


def test_symmetric_repeated_and_mirrored_entries(tmp_path):
    # (2,1) twice: both mirrored into (1,2); the diagonal kept once
    p = tmp_path / "rep.mtx"
    p.write_text("%%MatrixMarket matrix coordinate real symmetric\n3 3 5\n1 1 2.0\n2 1 -1\n3 3 5e0\n3 2 1.5\n2 1 0.25\n")
    got = read_matrix_market(p)
    assert np.array_equal(got[2], [0, 2, 4, 6]) and np.array_equal(got[3], [0, 1, 0, 2, 1, 2])
    assert np.array_equal(got[4], [2.0, -0.75, -0.75, 1.5, 1.5, 5.0])
    for want in _checkers(p):
        _same(got, want)


@pytest.mark.parametrize("field", ["pattern", "integer"])
def test_pattern_and_integer_fields(tmp_path, field):
    rng = np.random.default_rng(3)
    m = 50
    pairs = {(int(i), int(j)) for i, j in zip(rng.integers(0, m, 400), rng.integers(0, m, 400)) if j <= i}
    triples = [(i, j) if field == "pattern" else (i, j, int(rng.integers(-9, 10))) for i, j in sorted(pairs)]
    p = tmp_path / f"{field}.mtx"
    _write_triples(p, f"%%MatrixMarket matrix coordinate {field} symmetric", m, m, triples, fmt="{}")
    got = read_matrix_market(p)
    if field == "pattern":
        assert np.all(got[4] == 1.0)
    for want in _checkers(p):
        _same(got, want)


def test_banner_case_blank_lines_and_multithreaded_parse(tmp_path):
    A = M.grid_laplacian_3d(30, 5, 1e-2)           # 27,000 rows, ~100k stored entries
    p = tmp_path / "big.mtx"
    tr = _lower_triples(A)
    with open(p, "w") as f:
        f.write("%%MATRIXMARKET Matrix Coordinate REAL Symmetric\n% comment\n")
        f.write(f"{A.n} {A.n} {len(tr)}\n")
        for k, (i, j, v) in enumerate(tr):
            f.write(f"{i + 1}\t{j + 1}  {v:.17g}\r\n" + ("\n" if k % 997 == 0 else ""))
    one = read_matrix_market(p, thread_count=1)
    many = read_matrix_market(p, thread_count=8)
    _same(one, many)
    assert np.array_equal(one[4], A.values) and np.array_equal(one[3], A.inner)
    if oracle.ref_available():
        _same(one, oracle.ref_mm_read(p, 4))


def test_blank_line_before_the_size_line(tmp_path):
    # accepted here; the reference's comment loop (MatrixMarket.hpp:105-108)
    # stops at the blank line and reads a 0 x 0 size from it
    p = tmp_path / "blank.mtx"
    p.write_text("%%MatrixMarket matrix coordinate real general\n\n% c\n\n2 2 2\n1 1 1.5\n\n2 2 2.5\n")
    m, n, outer, inner, values = read_matrix_market(p)
    assert (m, n) == (2, 2) and np.array_equal(inner, [0, 1]) and np.array_equal(values, [1.5, 2.5])
    if oracle.ref_available():
        assert oracle.ref_mm_read(p)[0] == 0


REJECTED = {
    "not_mm": "%%Matrix matrix coordinate real general\n1 1 1\n1 1 1.0\n",
    "array": "%%MatrixMarket matrix array real general\n2 2\n1.0\n0.0\n0.0\n1.0\n",
    "complex": "%%MatrixMarket matrix coordinate complex general\n1 1 1\n1 1 1.0 0.0\n",
    "skew": "%%MatrixMarket matrix coordinate real skew-symmetric\n2 2 1\n2 1 1.0\n",
    "hermitian": "%%MatrixMarket matrix coordinate real hermitian\n1 1 1\n1 1 1.0\n",
    "bad_symmetry": "%%MatrixMarket matrix coordinate real upper\n1 1 1\n1 1 1.0\n",
    "not_matrix": "%%MatrixMarket vector coordinate real general\n1 1 1\n1 1 1.0\n",
}


@pytest.mark.parametrize("name", list(REJECTED))
def test_files_the_reference_rejects(tmp_path, name):
    p = tmp_path / f"{name}.mtx"
    p.write_text(REJECTED[name])
    with pytest.raises(TBError) as e:
        read_matrix_market(p)
    assert e.value.status == TB_ERR_FORMAT
    assert oracle.mm_read_port(p) is None
    if oracle.ref_available():
        assert oracle.ref_mm_read(p)[0] == 0       # the reference leaves the matrix empty


@pytest.mark.parametrize("body", [
    "3 3 1\n4 1 1.0\n",          # row index past the stated size
    "3 3 1\n1 0 1.0\n",          # zero index (files are 1-based)
    "3 3 2\n1 1 1.0\n",          # fewer entries than the size line states
    "3 3 1\n1 1 1.0\n2 2 1.0\n",  # more entries than it states
    "3 3 1\n1 1 x\n",            # malformed value
    "3 4 1\n1 1 1.0\n",          # symmetric but not square
])
def test_malformed_files_are_rejected(tmp_path, body):
    # the reference reads these past its buffers or into garbage; they are errors here
    p = tmp_path / "bad.mtx"
    p.write_text("%%MatrixMarket matrix coordinate real symmetric\n" + body)
    with pytest.raises(TBError) as e:
        read_matrix_market(p)
    assert e.value.status == TB_ERR_FORMAT


def test_missing_file(tmp_path):
    with pytest.raises(TBError) as e:
        read_matrix_market(tmp_path / "absent.mtx")
    assert e.value.status == TB_ERR_IO


def test_writer_text_and_bit_exact_round_trip(tmp_path):
    rng = np.random.default_rng(5)
    A = M.delaunay_laplacian(700, 2)
    bits = rng.integers(0, 2 ** 63, A.nnz, dtype=np.uint64) | (rng.integers(0, 2, A.nnz, dtype=np.uint64) << 63)
    vals = bits.view(np.float64).copy()
    vals[~np.isfinite(vals)] = 1.0
    vals[:3] = [0.0, -0.0, 5e-324]
    B = M.CSRMatrix(n=A.n, outer=A.outer, inner=A.inner, values=vals)
    p = tmp_path / "w.mtx"
    write_matrix_market(p, B)
    lines = p.read_text().splitlines()
    assert lines[0] == "%%MatrixMarket matrix coordinate real general"
    assert lines[1] == f"{A.n} {A.n} {A.nnz}"
    rows = np.repeat(np.arange(A.n), np.diff(A.outer))
    for k in (0, 1, 2, 17, A.nnz - 1):
        assert lines[2 + k] == f"{rows[k] + 1} {A.inner[k] + 1} {vals[k]:.17E}"   # C's "%d %d %.17E"
    got = read_matrix_market(p)
    _same(got, (A.n, A.n, A.outer, A.inner, vals))
    if oracle.ref_available():
        _same(got, oracle.ref_mm_read(p))


def test_rectangular_and_empty_matrices(tmp_path):
    p = tmp_path / "rect.mtx"
    write_matrix_market(p, (2, np.array([0, 1, 1]), np.array([4]), np.array([3.5])), cols=6)
    assert read_matrix_market(p)[:2] == (2, 6)
    with pytest.raises(ValueError):
        load_matrix_market(p)
    q = tmp_path / "empty.mtx"
    write_matrix_market(q, (3, np.zeros(4, np.int64), np.zeros(0, np.int32), np.zeros(0)))
    m, n, outer, inner, values = read_matrix_market(q)
    assert (m, n, len(inner), len(values)) == (3, 3, 0, 0) and np.array_equal(outer, [0, 0, 0, 0])


def test_loaded_matrix_gives_the_same_symbolic_structure(tmp_path):
    A = M.delaunay_laplacian(1500, 4)
    p = tmp_path / "mesh.mtx"
    _write_triples(p, "%%MatrixMarket matrix coordinate real symmetric", A.n, A.n, _lower_triples(A))
    B = load_matrix_market(p)
    perm = O.nested_dissection(A, 16)
    c1 = CholeskyDecomposition(A.outer, A.inner, perm)
    c2 = CholeskyDecomposition(B.outer, B.inner, perm)
    c1.SymbolicFactorization()
    c2.SymbolicFactorization()
    for key in ("perm", "value_perm", "SN_rp", "SN_outer", "SN_inner"):
        assert np.array_equal(c1.SymbolicArray(key), c2.SymbolicArray(key)), key


@pytest.mark.gpu
def test_factor_and_solve_a_matrix_read_from_a_file(tmp_path):
    A = M.grid_laplacian_3d(16, 8, 1e-3)
    p = tmp_path / "grid.mtx"
    _write_triples(p, "%%MatrixMarket matrix coordinate real symmetric", A.n, A.n, _lower_triples(A))
    B = load_matrix_market(p)
    c = CholeskyDecomposition(B.outer, B.inner, O.nested_dissection(A, 16))   # A: same matrix, with coordinates
    assert c.NumericFactorization(B.values) == 0
    rhs = np.random.default_rng(1).standard_normal((A.n, 3))
    X = c.Solve(rhs)
    R = rhs - M.csr_matvec(A, X)
    assert np.linalg.norm(R) <= 1e-12 * np.linalg.norm(rhs)


def test_binary_garbage_in_a_file_gives_a_status_not_a_decoding_error(tmp_path):
    # bytes that are not UTF-8 inside a malformed line and inside the banner
    p = tmp_path / "bin.mtx"
    p.write_bytes(b"%%MatrixMarket matrix coordinate real general\n2 2 1\n1 \xee\xff 1.0\n")
    with pytest.raises(TBError) as e:
        read_matrix_market(p)
    assert e.value.status == TB_ERR_FORMAT and "?" in str(e.value)
    p.write_bytes(b"%%MatrixMarket matrix coordinate r\xe9al general\n1 1 1\n1 1 1.0\n")
    with pytest.raises(TBError) as e:
        read_matrix_market(p)
    assert e.value.status == TB_ERR_FORMAT
