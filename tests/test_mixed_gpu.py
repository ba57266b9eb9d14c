"""Mixed precision: FP32 (optionally BF16-stored on the two finest levels)
hierarchy values and V-cycle arithmetic inside the FP64 PCG.  Every result is
checked against an FP64 oracle solve of the same system: the solve must still
reach the requested FP64 relative residual (the outer CG, its residual updates,
dot products and alpha/beta stay FP64), and the error against the FP64 oracle
solution is reported and bounded.
"""
import numpy as np
import pytest

from linalglib_b200 import _lib as L
from linalglib_b200 import problems as P

from helpers import inf_rel_residual

pytestmark = pytest.mark.gpu

CASES = {
    "poisson3d_24": lambda: P.poisson3d(24),
    "diffusion27_12": lambda: P.diffusion27(12, seed=0),
    "laplacian3d_16": lambda: P.graph_laplacian3d(16, seed=5),
}


@pytest.mark.parametrize("name", list(CASES))
@pytest.mark.parametrize("prec", [L.PREC_FP32, L.PREC_FP32_BF16])
def test_mixed_pcg_vs_fp64_oracle(gpu, oracle, name, prec):
    A = CASES[name]()
    b, _ = P.rhs_from_solution(*A, seed=0)
    dA = gpu.CsrMatrix.from_arrays(*A)
    H = gpu.Hierarchy(dA)
    ctl = gpu.iter_control(rel_tol=1e-10, abs_tol=0.0, max_iter=1000)
    M64 = gpu.Preconditioner.amg(H, gpu.amg_options(omega=2.0 / 3.0))
    x64, i64 = gpu.pcg(dA, gpu.vec(b), M=M64, control=ctl)
    Mlp = gpu.Preconditioner.amg(H, gpu.amg_options(omega=2.0 / 3.0, precision=prec))
    xlp, ilp = gpu.pcg(dA, gpu.vec(b), M=Mlp, control=ctl)
    xo, ito, _ = oracle.amg_setup(A).pcg(b, omega=2.0 / 3.0, coarse=1, rel_tol=1e-10, abs_tol=0.0,
                                         max_iter=1000)
    assert i64.converged and ilp.converged
    assert abs(i64.iterations - ito) <= 1
    # the low-precision preconditioner costs at most a few extra outer iterations
    slack = 3 if prec == L.PREC_FP32 else max(6, i64.iterations // 2)
    assert ilp.iterations <= i64.iterations + slack, (ilp.iterations, i64.iterations)
    xlp = xlp.cpu().numpy()
    assert inf_rel_residual(A, xlp, b) <= 1e-10 * 1.0001
    err = np.max(np.abs(xlp - xo)) / np.max(np.abs(xo))
    assert err <= 1e-7, err


@pytest.mark.parametrize("prec,tol", [(L.PREC_FP32, 1e-5), (L.PREC_FP32_BF16, 3e-2)])
def test_mixed_vcycle_close_to_fp64(gpu, prec, tol):
    A = P.poisson3d(20)
    dA = gpu.CsrMatrix.from_arrays(*A)
    H = gpu.Hierarchy(dA)
    r = gpu.vec(np.random.default_rng(0).uniform(-1, 1, A[0].size - 1))
    z64 = gpu.Preconditioner.amg(H).apply(r).cpu().numpy()
    zlp = gpu.Preconditioner.amg(H, gpu.amg_options(precision=prec)).apply(r).cpu().numpy()
    assert np.max(np.abs(zlp - z64)) <= tol * np.max(np.abs(z64))


def test_mixed_stationary_amg_refinement(gpu, oracle):
    """Stationary AMG in FP32 runs as iterative refinement x += V(0; b - A x)."""
    A = P.poisson2d(64)
    b, _ = P.rhs_from_solution(*A, seed=0)
    dA = gpu.CsrMatrix.from_arrays(*A)
    H = gpu.Hierarchy(dA)
    x, info = H.solve(gpu.vec(b), options=gpu.amg_options(precision=L.PREC_FP32),
                      control=gpu.iter_control(rel_tol=1e-9, abs_tol=0.0, max_cycle=400))
    xo, ito = oracle.amg_setup(A).amg_solve(b, coarse=1, rel_tol=1e-9, abs_tol=0.0, max_cycle=400)
    assert info.converged
    assert abs(info.iterations - ito) <= 2
    assert np.max(np.abs(x.cpu().numpy() - xo)) <= 1e-7 * np.max(np.abs(xo))


def test_mixed_gmres(gpu):
    A = P.diffusion27(10, seed=2)
    b, _ = P.rhs_from_solution(*A, seed=0)
    dA = gpu.CsrMatrix.from_arrays(*A)
    H = gpu.Hierarchy(dA)
    M = gpu.Preconditioner.amg(H, gpu.amg_options(omega=2.0 / 3.0, precision=L.PREC_FP32))
    x, info = gpu.gmres(dA, gpu.vec(b), M=M, restart=40,
                        control=gpu.iter_control(rel_tol=1e-10, abs_tol=0.0, max_iter=100))
    assert info.converged
    assert inf_rel_residual(A, x.cpu().numpy(), b) <= 1e-8
