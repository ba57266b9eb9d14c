"""Halo form of the VECTOR schedule (k_vhalo, LAB_SPMV_VECTOR_HALO): x staged per
chunk of consecutive rows at the chunk's distinct columns in shared memory.

* the plan: the default analysis builds none; forced on the coarse SA operators of
  a 3D Poisson hierarchy, the chunks and their distinct-column counts (against
  numpy's unique per chunk) and the schedule reported;
* bit-identity: SpMV (alpha, beta), residual and whole V-cycles in FP64, FP32 and
  FP32 + BF16 equal the direct-load kernel (same lanes, same order per row);
* chunks whose column span exceeds the bitmap read x directly, next to staged
  chunks, and integer-valued data gives numpy's exact result;
* a halo on a matrix without column locality still gives the direct results.
"""
import numpy as np
import pytest

from linalglib_b200 import _lib as L
from linalglib_b200 import problems as P

pytestmark = pytest.mark.gpu


def _bits(a):
    return np.ascontiguousarray(a).view(np.int64)


def _exact_spmv(rp, ci, v, x):
    rows = np.repeat(np.arange(rp.size - 1), np.diff(rp))
    y = np.zeros(rp.size - 1)
    np.add.at(y, rows, v * x[ci])
    return y


@pytest.fixture(scope="module")
def poisson64(gpu):
    A = P.poisson3d(64)
    dA = gpu.CsrMatrix.from_arrays(*A)
    H = gpu.Hierarchy(dA)
    return A, dA, H


def test_halo_plan_and_bit_identity_on_sa_levels(gpu, poisson64):
    _, _, H = poisson64
    rng = np.random.default_rng(3)
    built = 0
    for l in range(1, H.levels + 1):
        M = H.A(l)
        M.analyse()
        m, n, nnz = M.info()
        alg, w = M.algorithm()
        assert M.halo_info() == (0, 0, 0, 0) and alg != L.SPMV_VECTOR_HALO
        if alg != L.SPMV_VECTOR:
            continue
        M.set_algorithm(L.SPMV_VECTOR_HALO, w)
        chunks, rows, distinct, direct = M.halo_info()
        assert M.algorithm() == (L.SPMV_VECTOR_HALO, w) and chunks > 0, l
        rp, ci = M.to_numpy()[:2]
        uniq = [np.unique(ci[rp[r]:rp[min(m, r + rows)]]).size for r in range(0, m, rows)]
        assert chunks == len(uniq) and direct == 0
        assert distinct == sum(uniq)
        if nnz > 32 * m:  # long rows near the diagonal: far fewer columns than entries
            assert distinct <= 0.6 * nnz
            built += 1
        x = gpu.vec(rng.uniform(-1, 1, n))
        y0 = rng.uniform(-1, 1, m)
        b = gpu.vec(rng.uniform(-1, 1, m))
        yh = M.spmv(x, gpu.vec(y0), alpha=1.5, beta=-0.5).cpu().numpy()
        rh = M.residual(x, b).cpu().numpy()
        M.set_algorithm(L.SPMV_VECTOR, w)
        assert M.algorithm() == (L.SPMV_VECTOR, w)
        yd = M.spmv(x, gpu.vec(y0), alpha=1.5, beta=-0.5).cpu().numpy()
        rd = M.residual(x, b).cpu().numpy()
        assert np.array_equal(_bits(yh), _bits(yd)), l
        assert np.array_equal(_bits(rh), _bits(rd)), l
        for lanes in (4, 16):  # other lane counts over the same chunks
            M.set_algorithm(L.SPMV_VECTOR_HALO, lanes)
            assert M.algorithm() == (L.SPMV_VECTOR_HALO, lanes)
            yh = M.spmv(x).cpu().numpy()
            M.set_algorithm(L.SPMV_VECTOR, lanes)
            assert np.array_equal(_bits(yh), _bits(M.spmv(x).cpu().numpy())), (l, lanes)
        M.set_algorithm(L.SPMV_VECTOR, w)  # the level's own schedule; the plan stays
        assert M.algorithm() == (L.SPMV_VECTOR, w)
        assert M.halo_info()[0] == chunks
    assert built >= 2
    # prolongations and restrictions are rectangular: no halo plan
    for l in range(H.levels):
        for X in (H.P(l), H.R(l)):
            X.analyse()
            assert X.halo_info()[0] == 0


@pytest.mark.parametrize("prec", [L.PREC_FP64, L.PREC_FP32, L.PREC_FP32_BF16])
def test_halo_cycle_equals_direct(gpu, poisson64, prec):
    """A V-cycle whose coarse operators run the halo form equals the cycle with
    every coarse pass reading x directly, bit for bit."""
    A, _, H = poisson64
    r = gpu.vec(np.random.default_rng(1).uniform(-1, 1, A[0].size - 1))
    mats = [H.A(l) for l in range(1, H.levels + 1)]
    vec = [(M, M.algorithm()[1]) for M in mats if M.algorithm()[0] == L.SPMV_VECTOR]
    assert vec
    Mp = gpu.Preconditioner.amg(H, gpu.amg_options(precision=prec))
    z_direct = Mp.apply(r).cpu().numpy()
    for M, w in vec:
        M.set_algorithm(L.SPMV_VECTOR_HALO, w)
        assert M.algorithm()[0] == L.SPMV_VECTOR_HALO
    z_halo = Mp.apply(r).cpu().numpy()
    for M, w in vec:
        M.set_algorithm(L.SPMV_VECTOR, w)
    assert np.array_equal(_bits(z_halo), _bits(z_direct))


def _banded(m, rng, far_every):
    """Square matrix, ~40 entries per row at offsets within +-60 of the diagonal
    (one of 64 random offset patterns per row), integer values; every far_every-th
    row also has entries in columns 0 and m - 1."""
    pats = [np.sort(rng.choice(121, size=40, replace=False)) - 60 for _ in range(64)]
    pick = rng.integers(0, 64, size=m)
    rows, cols = [], []
    for k in range(64):
        rr = np.nonzero(pick == k)[0]
        c = rr[:, None] + pats[k][None, :]
        rows.append(np.repeat(rr, pats[k].size))
        cols.append(c.ravel())
    far = np.arange(0, m, far_every)
    rows += [far, far]
    cols += [np.zeros(far.size, dtype=np.int64), np.full(far.size, m - 1)]
    rows = np.concatenate(rows)
    cols = np.concatenate(cols)
    keep = (cols >= 0) & (cols < m)
    key = np.unique(rows[keep].astype(np.int64) * m + cols[keep])
    r, c = key // m, key % m
    rp = np.zeros(m + 1, dtype=np.int64)
    np.add.at(rp, r + 1, 1)
    rp = np.cumsum(rp).astype(np.int32)
    v = rng.integers(-3, 4, size=c.size).astype(np.float64)
    return rp, c.astype(np.int32), v


def test_halo_direct_chunks_and_exact_integers(gpu):
    rng = np.random.default_rng(11)
    m = 400_000
    rp, ci, v = _banded(m, rng, far_every=20_000)
    x = rng.integers(-4, 5, size=m).astype(np.float64)
    bb = rng.integers(-4, 5, size=m).astype(np.float64)
    A = gpu.CsrMatrix.from_arrays(rp, ci, v)
    A.analyse()
    alg, w = A.algorithm()
    assert alg == L.SPMV_VECTOR
    A.set_algorithm(L.SPMV_VECTOR_HALO, w)
    chunks, rows, distinct, direct = A.halo_info()
    assert A.algorithm() == (L.SPMV_VECTOR_HALO, w)
    # the chunks holding a row with columns 0 and m - 1 span more than the bitmap
    assert direct == np.unique(np.arange(0, m, 20_000) // rows).size
    assert 0 < direct < chunks
    y_exact = _exact_spmv(rp, ci, v, x)
    y = A.spmv(gpu.vec(x)).cpu().numpy()
    assert np.array_equal(y, y_exact)
    r = A.residual(gpu.vec(x), gpu.vec(bb)).cpu().numpy()
    assert np.array_equal(r, bb - y_exact)
    A.set_algorithm(L.SPMV_VECTOR, w)
    assert np.array_equal(A.spmv(gpu.vec(x)).cpu().numpy(), y_exact)


def test_halo_without_locality(gpu):
    """Random columns over the whole matrix: a halo saves few gathers but still
    gives the direct kernel's results bit for bit."""
    rng = np.random.default_rng(5)
    m = 60_000
    rows = np.repeat(np.arange(m), rng.poisson(41, size=m))
    key = np.unique(rows.astype(np.int64) * m + rng.integers(0, m, size=rows.size))
    rp = np.zeros(m + 1, dtype=np.int64)
    np.add.at(rp, key // m + 1, 1)
    rp = np.cumsum(rp).astype(np.int32)
    ci = (key % m).astype(np.int32)
    v = rng.uniform(-1, 1, ci.size)
    x = gpu.vec(rng.uniform(-1, 1, m))
    A = gpu.CsrMatrix.from_arrays(rp, ci, v)
    A.analyse()
    assert A.halo_info()[0] == 0 and A.algorithm()[0] == L.SPMV_VECTOR
    y_direct = A.spmv(x).cpu().numpy()
    B = gpu.CsrMatrix.from_arrays(rp, ci, v)
    B.set_algorithm(L.SPMV_VECTOR_HALO, A.algorithm()[1])
    chunks, rows, distinct, direct = B.halo_info()
    assert chunks > 0 and B.algorithm()[0] == L.SPMV_VECTOR_HALO
    assert distinct > 0.6 * ci.size
    assert np.array_equal(_bits(B.spmv(x).cpu().numpy()), _bits(y_direct))
