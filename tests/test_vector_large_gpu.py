"""VECTOR SpMV (W lanes per row, every W) on matrices of 1-1.6 M entries.
Integer-valued matrices and vectors make every summation order exact, so an
indexing slip (lane-strided entries, row ends, rows of up to 4000 entries
between short ones, empty rows) shows as a difference from numpy;
real-valued cases follow the reference's SpMV acceptance bound
(clients/common/utility.cpp:526-544)."""
import numpy as np
import pytest

from linalglib_b200 import _lib as L

pytestmark = pytest.mark.gpu


def _csr_from_lens(lens, n, rng, ints):
    m = lens.size
    rp = np.zeros(m + 1, dtype=np.int64)
    np.cumsum(lens, out=rp[1:])
    nnz = int(rp[-1])
    # sorted distinct columns per row: a random start and strictly increasing gaps
    gaps = rng.integers(1, 4, size=nnz)
    starts = np.repeat(np.arange(m), lens)
    first = np.zeros(nnz, dtype=bool)
    first[rp[:-1][lens > 0]] = True
    gaps[first] = 0
    seg = np.cumsum(gaps)
    seg -= np.repeat(seg[rp[:-1]], lens) if nnz else seg
    base = rng.integers(0, n, size=m)
    ci = (np.repeat(base, lens) + seg) % n
    # keep each row sorted after the wrap-around
    order = np.lexsort((ci, starts))
    ci = ci[order]
    if ints:
        v = rng.integers(-3, 4, size=nnz).astype(np.float64)
    else:
        v = rng.uniform(-1, 1, size=nnz)
    return rp.astype(np.int32), ci.astype(np.int32), v


def _dense_ref(rp, ci, v, x):
    rows = np.repeat(np.arange(rp.size - 1), np.diff(rp))
    y = np.zeros(rp.size - 1)
    np.add.at(y, rows, v * x[ci])
    return y


CASES = {
    # mean 41 (an SA level-1 operator's rows), Poisson lengths, some empty rows
    "mean41": lambda rng: rng.poisson(41, size=40000),
    # mean 143 with a wide spread
    "mean143": lambda rng: rng.integers(0, 290, size=9000),
    # short rows with a long row every 997 rows
    "spiky": lambda rng: np.where(np.arange(150000) % 997 == 5, 4000, rng.poisson(6, size=150000)),
    # rows of ~1000 entries
    "long": lambda rng: rng.integers(900, 1100, size=1100),
}


@pytest.mark.parametrize("case", list(CASES))
@pytest.mark.parametrize("lanes", [2, 4, 8, 16, 32])
def test_vector_exact_on_integers(gpu, case, lanes):
    rng = np.random.default_rng(lanes * 31 + len(case))
    lens = CASES[case](rng).astype(np.int64)
    n = 50000
    lens = np.minimum(lens, n // 4)
    rp, ci, v = _csr_from_lens(lens, n, rng, ints=True)
    assert rp[-1] >= 1 << 20
    x = rng.integers(-4, 5, size=n).astype(np.float64)
    y0 = rng.integers(-4, 5, size=rp.size - 1).astype(np.float64)
    A = gpu.CsrMatrix.from_arrays(rp, ci, v, n=n)
    A.set_algorithm(L.SPMV_VECTOR, lanes)
    y = A.spmv(gpu.vec(x), gpu.vec(y0), alpha=2.0, beta=-1.0).cpu().numpy()
    assert np.array_equal(y, 2.0 * _dense_ref(rp, ci, v, x) - y0)


@pytest.mark.parametrize("lanes", [4, 8, 16])
def test_vector_matches_oracle(gpu, oracle, lanes):
    rng = np.random.default_rng(5 + lanes)
    lens = rng.poisson(41, size=30000).astype(np.int64)
    n = 30000
    rp, ci, v = _csr_from_lens(lens, n, rng, ints=False)
    x = rng.uniform(-1, 1, n)
    A = gpu.CsrMatrix.from_arrays(rp, ci, v, n=n)
    A.set_algorithm(L.SPMV_VECTOR, lanes)
    y = A.spmv(gpu.vec(x)).cpu().numpy()
    yo = oracle.spmv((rp, ci, v, n), x)
    assert np.max(np.abs(y - yo)) <= 1e-9
    # deterministic: a second run is identical
    assert np.array_equal(A.spmv(gpu.vec(x)).cpu().numpy(), y)
