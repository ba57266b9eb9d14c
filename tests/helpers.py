"""Shared comparison predicates for the parity tests."""
import numpy as np


def bits_equal(a, b):
    """Bitwise equality of float arrays, treating any NaN as equal to any NaN.

    IEEE 754 leaves the sign and payload of a NaN produced by arithmetic
    unspecified, and compilers may reorder a negation around it (the reference's
    0/0 in RS direct interpolation, rsamg.cpp:838-839, is the one place a NaN
    appears).
    """
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    if a.shape != b.shape:
        return False
    na, nb = np.isnan(a), np.isnan(b)
    if not np.array_equal(na, nb):
        return False
    return np.array_equal(a[~na].view(np.int64), b[~nb].view(np.int64))


def csr_equal(x, y):
    """(rp, ci, v, n) tuples identical: pattern exact, values bitwise (NaN ~ NaN)."""
    if x[3] != y[3]:
        return False
    return (np.array_equal(x[0], y[0]) and np.array_equal(x[1], y[1]) and bits_equal(x[2], y[2]))


def csr_diff(x, y):
    """Human-readable first difference between two CSR tuples."""
    if x[3] != y[3]:
        return f"n {x[3]} != {y[3]}"
    if x[0].shape != y[0].shape:
        return f"m {x[0].size - 1} != {y[0].size - 1}"
    d = np.nonzero(x[0] != y[0])[0]
    if d.size:
        return f"row_ptr differs at {d[0]}: {x[0][d[0]]} vs {y[0][d[0]]}"
    if x[1].shape != y[1].shape:
        return "nnz differs"
    d = np.nonzero(x[1] != y[1])[0]
    if d.size:
        return f"col_ind differs at {d[0]}: {x[1][d[0]]} vs {y[1][d[0]]}"
    d = np.nonzero(x[2].view(np.int64) != y[2].view(np.int64))[0]
    if d.size:
        return f"{d.size} values differ, first at {d[0]}: {x[2][d[0]]!r} vs {y[2][d[0]]!r}"
    return "equal"


def inf_rel_residual(A, x, b):
    """||b - A x||_inf / ||b||_inf on the host (float64)."""
    rp, ci, v = A[0], A[1], A[2]
    m = rp.size - 1
    rows = np.repeat(np.arange(m), np.diff(rp))
    ax = np.bincount(rows, weights=v * x[ci], minlength=m)
    return np.max(np.abs(b - ax)) / np.max(np.abs(b))
