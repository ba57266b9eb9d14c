"""Matrix Market I/O (lab_mtx_read / lab_mtx_write, behind csr_matrix::read_mtx /
write_mtx) against the reference's own csr_matrix::read_mtx / write_mtx
(library/src/csr_matrix.cpp:523-795) compiled into oracle/_ref.  Host-only code:
these tests need no GPU.

* reading: the CSR arrays are bit-identical to the reference's on general,
  symmetric and integer files with comments and repeated entries (summed in the
  reference's order), and every file the reference refuses is refused;
* writing: the two files are identical byte for byte;
* files the reference would crash on (an index outside the stated size, an
  entry line without its fields) are refused here and not given to the
  reference.
"""
import zlib

import numpy as np
import pytest

from linalglib_b200 import _lib as L

from helpers import csr_diff, csr_equal


def _write(path, text):
    path.write_text(text)
    return path


def _random_entries(rng, m, n, count, dups):
    rows = rng.integers(1, m + 1, size=count)
    cols = rng.integers(1, n + 1, size=count)
    # repeat some positions several times with values of very different size, so
    # a different summation order would change the bits
    k = rng.integers(0, count, size=dups)
    rows = np.concatenate([rows, np.repeat(rows[k], 3)])
    cols = np.concatenate([cols, np.repeat(cols[k], 3)])
    vals = rng.standard_normal(rows.size) * 10.0 ** rng.integers(-8, 9, size=rows.size)
    perm = rng.permutation(rows.size)
    return rows[perm], cols[perm], vals[perm]


def _mtx_text(kind, sym, m, n, rows, cols, vals, comments=2, fmt="{:.17g}"):
    lines = [f"%%MatrixMarket matrix coordinate {kind} {sym}"]
    lines += [f"% comment {c}" for c in range(comments)]
    lines.append(f"{m} {n} {rows.size}")
    for r, c, v in zip(rows, cols, vals):
        lines.append(f"{r} {c} {fmt.format(v)}")
    return "\n".join(lines) + "\n"


@pytest.mark.parametrize("case", ["general", "general_rect", "symmetric", "integer", "empty",
                                  "crlf", "no_trailing_newline"])
def test_read_mtx_matches_reference(reference, tmp_path, case):
    rng = np.random.default_rng(zlib.crc32(case.encode()))
    m, n = (40, 40) if case != "general_rect" else (30, 55)
    rows, cols, vals = _random_entries(rng, m, n, 300, 40)
    kind, sym, fmt = "real", "general", "{:.17g}"
    if case == "symmetric":
        sym = "symmetric"
        keep = rows >= cols  # lower triangle, as symmetric files store it
        rows, cols, vals = rows[keep], cols[keep], vals[keep]
    if case == "integer":
        kind, fmt = "integer", "{:.0f}"
        vals = np.round(vals / 1e4)
    if case == "empty":
        rows, cols, vals = rows[:0], cols[:0], vals[:0]
    text = _mtx_text(kind, sym, m, n, rows, cols, vals, fmt=fmt)
    if case == "crlf":
        text = text.replace("\n", "\r\n")
    if case == "no_trailing_newline":
        text = text.rstrip("\n")
    p = _write(tmp_path / "a.mtx", text)
    ours = L.mtx_read(p)
    ref = reference.read_mtx(p)
    assert ref is not None
    assert csr_equal(ours, ref), csr_diff(ours, ref)
    if case != "empty":
        assert ours[2].size < rows.size * (2 if sym == "symmetric" else 1)  # duplicates merged


@pytest.mark.parametrize("banner", [
    "%%MatrixMarket matrix array real general",
    "%%MatrixMarket matrix coordinate complex general",
    "%%MatrixMarket matrix coordinate pattern general",
    "%%MatrixMarket matrix coordinate real hermitian",
    "%%MatrixMarket matrix coordinate real skew-symmetric",
    "%%MatrixMarket vector coordinate real general",
    "%%MatrixMarket matrix coordinate real",
    "%%MatrixMarket matrix coordinate",
    "",
])
def test_read_mtx_refuses_what_the_reference_refuses(reference, tmp_path, banner):
    body = "3 3 2\n1 1 1.5\n2 3 -2.0\n"
    p = _write(tmp_path / "r.mtx", banner + "\n" + body)
    assert reference.read_mtx(p) is None
    with pytest.raises(L.LabError):
        L.mtx_read(p)


@pytest.mark.parametrize("body", [
    "3 3 1\n4 1 1.0\n",    # row beyond m: the reference writes outside its row pointer
    "3 3 1\n0 1 1.0\n",    # row 0 in a 1-based file
    "3 3 1\n1 9 1.0\n",    # column beyond n
    "3 3 2\n1 1 1.0\n",    # fewer entries than stated
    "3 3 1\n1  1 1.0\n",   # an empty column field (std::stoi would throw)
    "-3 3 0\n",            # negative size
])
def test_read_mtx_refuses_broken_files(tmp_path, body):
    p = _write(tmp_path / "b.mtx", "%%MatrixMarket matrix coordinate real general\n" + body)
    with pytest.raises(L.LabError):
        L.mtx_read(p)


def test_read_mtx_missing_file(tmp_path):
    with pytest.raises(L.LabError):
        L.mtx_read(tmp_path / "none.mtx")


@pytest.mark.parametrize("shape", [(25, 25), (12, 31), (0, 0)])
def test_write_mtx_bytes_match_reference(reference, tmp_path, shape):
    m, n = shape
    rng = np.random.default_rng(m * 100 + n)
    dense = rng.standard_normal((m, n)) * 10.0 ** rng.integers(-12, 6, size=(m, n))
    dense[rng.random((m, n)) < 0.7] = 0.0
    if m:
        dense[0, 0] = -0.0
        dense[-1, -1] = 123456789.0123456789
    rows, cols = np.nonzero(dense != 0.0) if m else (np.zeros(0, int), np.zeros(0, int))
    rp = np.zeros(m + 1, dtype=np.int32)
    np.add.at(rp, rows + 1, 1)
    rp = np.cumsum(rp).astype(np.int32)
    A = (rp, cols.astype(np.int32), dense[rows, cols], n)
    L.mtx_write(tmp_path / "ours.mtx", *A)
    assert reference.write_mtx(tmp_path / "ref.mtx", A)
    assert (tmp_path / "ours.mtx").read_bytes() == (tmp_path / "ref.mtx").read_bytes()
    # and the written file reads back to the same pattern (values rounded to 10 decimals)
    back = L.mtx_read(tmp_path / "ours.mtx")
    assert np.array_equal(back[0], rp) or m == 0
