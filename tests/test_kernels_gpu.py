"""CUDA kernels vs the oracle: SpMV (both schedules), residual, BLAS-1, scans.

Acceptance predicates follow the reference tests: SpMV |dy| <= 1e-9
(clients/common/utility.cpp:526-544), and bit-exact where the arithmetic order is
the reference's (staged thread-per-row SpMV with fma in CSR order, residual,
axpy/axpby/axpbypgz, integer scans).
"""
import numpy as np
import pytest
import torch

from linalglib_b200 import _lib as L
from linalglib_b200 import problems as P

pytestmark = pytest.mark.gpu


def _rand_csr(m, n, avg, seed, maxlen=None):
    rng = np.random.default_rng(seed)
    lens = rng.poisson(avg, size=m)
    if maxlen is not None:
        lens = np.minimum(lens, maxlen)
    lens = np.minimum(lens, n)
    rp = np.zeros(m + 1, dtype=np.int32)
    np.cumsum(lens, out=rp[1:])
    ci = np.concatenate([np.sort(rng.choice(n, size=k, replace=False)) for k in lens]).astype(np.int32) \
        if rp[-1] else np.zeros(0, np.int32)
    v = rng.uniform(-1, 1, size=rp[-1])
    return rp, ci, v, n


MATS = {
    "poisson2d_64": lambda: (*P.poisson2d(64), 64 * 64),
    "poisson3d_24": lambda: (*P.poisson3d(24), 24 ** 3),
    "random_short": lambda: _rand_csr(5000, 4000, 5.0, 1, maxlen=16),
    "random_long": lambda: _rand_csr(3000, 6000, 60.0, 2),
    "random_skewed": lambda: _rand_csr(2000, 2000, 3.0, 3),
    "empty_rows": lambda: (np.array([0, 0, 2, 2, 3], np.int32), np.array([0, 3, 1], np.int32),
                           np.array([1.0, 2.0, 3.0]), 4),
}


@pytest.mark.parametrize("name", list(MATS))
@pytest.mark.parametrize("alg", [L.SPMV_AUTO, L.SPMV_ROWSEQ, L.SPMV_VECTOR])
@pytest.mark.parametrize("alpha,beta", [(1.0, 0.0), (1.0, 1.0), (-0.5, 2.0)])
def test_spmv_matches_oracle(gpu, oracle, name, alg, alpha, beta):
    rp, ci, v, n = MATS[name]()
    m = rp.size - 1
    rng = np.random.default_rng(1234567)
    x = rng.uniform(-1, 1, n)
    y0 = rng.uniform(-1, 1, m)
    A = gpu.CsrMatrix.from_arrays(rp, ci, v, n=n)
    if alg != L.SPMV_AUTO:
        A.set_algorithm(alg, 8 if alg == L.SPMV_VECTOR else 0)
    y = A.spmv(gpu.vec(x), gpu.vec(y0), alpha=alpha, beta=beta).cpu().numpy()
    yo = oracle.spmv((rp, ci, v, n), x, alpha=alpha, beta=beta, y=y0)
    assert np.max(np.abs(y - yo), initial=0.0) <= 1e-9
    if A.algorithm()[0] == L.SPMV_ROWSEQ:
        # fma in CSR order: bit-identical to host_csrmv_impl
        assert np.array_equal(y.view(np.int64), yo.view(np.int64))


def test_spmv_matches_reference_bitwise(gpu, reference):
    rp, ci, v = P.poisson3d(20)
    x = np.random.default_rng(0).uniform(-1, 1, rp.size - 1)
    A = gpu.CsrMatrix.from_arrays(rp, ci, v)
    y = A.spmv(gpu.vec(x)).cpu().numpy()
    yr = reference.spmv((rp, ci, v), x)
    assert np.array_equal(y.view(np.int64), yr.view(np.int64))


@pytest.mark.parametrize("name", ["poisson2d_64", "random_long", "empty_rows"])
def test_residual_bitwise(gpu, oracle, name):
    rp, ci, v, n = MATS[name]()
    m = rp.size - 1
    rng = np.random.default_rng(7)
    x, b = rng.uniform(-1, 1, n), rng.uniform(-1, 1, m)
    A = gpu.CsrMatrix.from_arrays(rp, ci, v, n=n)
    A.set_algorithm(L.SPMV_ROWSEQ)
    r = A.residual(gpu.vec(x), gpu.vec(b)).cpu().numpy()
    ro = oracle.residual((rp, ci, v, n), x, b)
    assert np.array_equal(r.view(np.int64), ro.view(np.int64))


def test_spmv_deterministic(gpu):
    rp, ci, v, n = _rand_csr(20000, 20000, 40.0, 9)
    A = gpu.CsrMatrix.from_arrays(rp, ci, v, n=n)
    x = gpu.vec(np.random.default_rng(3).uniform(-1, 1, n))
    y1 = A.spmv(x).clone()
    y2 = A.spmv(x)
    assert torch.equal(y1, y2)


def test_blas1(gpu):
    rng = np.random.default_rng(11)
    n = 1_000_003
    x, y, z = (rng.uniform(-1, 1, n) for _ in range(3))
    tx, ty, tz = gpu.vec(x), gpu.vec(y), gpu.vec(z)
    d = gpu.dot(tx, ty)
    assert abs(d - np.dot(x, y)) <= 1e-12 * n
    assert gpu.dot(tx, ty) == d  # deterministic
    assert gpu.norm_inf(tx) == np.max(np.abs(x))
    assert abs(gpu.norm_euclid(tx) - np.linalg.norm(x)) <= 1e-12 * np.linalg.norm(x)
    gpu.axpy(0.25, tx, ty)
    ref = 0.25 * x + y
    assert np.array_equal(ty.cpu().numpy(), ref)
    gpu.axpby(1.5, tx, -0.5, tz)
    refz = 1.5 * x + (-0.5) * z
    assert np.array_equal(tz.cpu().numpy(), refz)
    gpu.axpbypgz(1.0, tx, 2.0, ty, 3.0, tz)
    assert np.array_equal(tz.cpu().numpy(), 1.0 * x + 2.0 * ref + 3.0 * refz)


@pytest.mark.parametrize("n", [0, 1, 7, 2048, 2049, 1_000_000])
@pytest.mark.parametrize("dtype", [torch.int32, torch.int64])
def test_exclusive_scan(gpu, n, dtype):
    rng = np.random.default_rng(n)
    a = rng.integers(0, 5, size=n)
    t = torch.as_tensor(a, dtype=dtype, device="cuda")
    gpu.exclusive_scan(t)
    ref = np.concatenate([[0], np.cumsum(a)[:-1]]) if n else a
    assert np.array_equal(t.cpu().numpy(), ref)


def test_diagonal_and_spmm(gpu, oracle):
    rp, ci, v = P.poisson2d(40)
    A = gpu.CsrMatrix.from_arrays(rp, ci, v)
    assert torch.equal(A.diagonal().cpu(), torch.full((1600,), 4.0, dtype=torch.float64))
    rng = np.random.default_rng(5)
    X = rng.uniform(-1, 1, (11, 1600))
    Y = A.spmm(gpu.vec(X).reshape(11, 1600)).cpu().numpy()
    for k in range(11):
        assert np.max(np.abs(Y[k] - oracle.spmv((rp, ci, v), X[k]))) <= 1e-12


def test_bad_csr_rejected(gpu):
    with pytest.raises(L.LabError):
        gpu.CsrMatrix.from_arrays(np.array([0, 2, 1], np.int32), np.array([0, 1], np.int32),
                                  np.array([1.0, 2.0]))
    with pytest.raises(L.LabError):
        gpu.CsrMatrix.from_arrays(np.array([0, 1], np.int32), np.array([5], np.int32),
                                  np.array([1.0]))
