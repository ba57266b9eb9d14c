"""SpMV schedule autotuner: the tuned plan is one of the candidates, an exact tune
keeps results bit-identical to the reference-order SpMV, a free tune stays within
the vector-schedule tolerance, and a tuned hierarchy still solves like the oracle."""
import numpy as np
import pytest

from linalglib_b200 import _lib as L
from linalglib_b200 import problems as P

pytestmark = pytest.mark.gpu

CASES = {
    "poisson3d_32": lambda: P.poisson3d(32),
    "diffusion27_20": lambda: P.diffusion27(20, seed=1),
}


@pytest.mark.parametrize("name", list(CASES))
def test_spmv_autotune_keeps_results(gpu, oracle, name):
    A = CASES[name]()
    x = np.random.default_rng(0).uniform(-1, 1, A[0].size - 1)
    y_ref = oracle.spmv(A, x)  # reference order (fma in CSR order)
    dA = gpu.CsrMatrix.from_arrays(*A)
    us = dA.autotune(exact=True)
    assert us > 0
    assert dA.algorithm()[0] == L.SPMV_ROWSEQ
    y = dA.spmv(gpu.vec(x)).cpu().numpy()
    assert np.array_equal(y, y_ref)
    dA.autotune(exact=False)
    alg, lanes = dA.algorithm()
    assert (alg, lanes) in [(L.SPMV_ROWSEQ, 1)] + [(a, w) for w in (2, 4, 8, 16, 32)
                                                   for a in (L.SPMV_VECTOR, L.SPMV_VECTOR_STREAM,
                                                             L.SPMV_VECTOR_HALO)]
    y = dA.spmv(gpu.vec(x)).cpu().numpy()
    assert np.max(np.abs(y - y_ref)) <= 1e-9


def test_hierarchy_autotune_solves_like_oracle(gpu, oracle):
    A = P.poisson3d(24)
    b, _ = P.rhs_from_solution(*A, seed=0)
    dA = gpu.CsrMatrix.from_arrays(*A)
    H = gpu.Hierarchy(dA)
    H.autotune(exact=False)
    M = gpu.Preconditioner.amg(H, gpu.amg_options(omega=2.0 / 3.0))
    x, info = gpu.pcg(dA, gpu.vec(b), M=M,
                      control=gpu.iter_control(rel_tol=1e-8, abs_tol=0.0, max_iter=200))
    xo, ito, _ = oracle.amg_setup(A).pcg(b, omega=2.0 / 3.0, coarse=1, rel_tol=1e-8, abs_tol=0.0,
                                         max_iter=200)
    assert info.converged == 1
    assert abs(info.iterations - ito) <= 1
    assert np.max(np.abs(x.cpu().numpy() - xo)) <= 1e-6 * np.max(np.abs(xo))


def test_spgemm_autotune_keeps_results(gpu, oracle):
    """Tuning only sizes the hash tables: the products stay bit-identical."""
    import ctypes as C
    from helpers import csr_equal
    A = P.poisson3d(24)
    Ho = oracle.amg_setup(A)
    dA = gpu.CsrMatrix.from_arrays(*A)
    dP = gpu.CsrMatrix.from_arrays(*Ho.P(0)[:3], n=Ho.P(0)[3])
    before = dA.spgemm(dP).to_numpy()
    us = C.c_double()
    L.call("lab_spgemm_autotune", dA.h, dP.h, C.byref(us), gpu.stream_handle())
    assert us.value > 0
    after = dA.spgemm(dP).to_numpy()
    assert csr_equal(before, after)
    assert csr_equal(after, oracle.spgemm(A, Ho.P(0)))


def test_hierarchy_tune_products_then_setup_bit_identical(gpu, oracle):
    """After the Galerkin products of a hierarchy are tuned, a new setup of the same
    operator uses the tuned sizings and is still bit-identical to the oracle."""
    from helpers import csr_equal
    A = P.poisson3d(20)
    dA = gpu.CsrMatrix.from_arrays(*A)
    H = gpu.Hierarchy(dA)
    L.call("lab_hierarchy_tune_products", H.h, gpu.stream_handle())
    H2 = gpu.Hierarchy(dA)
    Ho = oracle.amg_setup(A)
    assert H2.levels == Ho.levels
    for l in range(H2.levels + 1):
        assert csr_equal(H2.A(l).to_numpy(), Ho.A(l))
    L.call("lab_tune_cache_clear")
