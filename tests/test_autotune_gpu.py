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
                                                   for a in (L.SPMV_VECTOR, L.SPMV_VECTOR_STREAM)]
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
