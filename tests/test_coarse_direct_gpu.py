"""Dense direct coarsest solve (LAB_COARSE_DIRECT) on coarsest levels of 159 to 1515
rows (hierarchies cut short by max_level): the Gauss-Jordan inverse -- one CTA up to
256 rows, else one pivot kernel and one elimination pass over the GPU per column --
against the oracle's Gauss-Jordan inverse (oracle.c build_coarse_inverse), through
the V-cycle and the PCG solve."""
import numpy as np
import pytest

from linalglib_b200 import _lib as L
from linalglib_b200 import problems as P

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("n, ml, nc", [(36, 2, 1515), (28, 2, 743), (16, 2, 159)])
def test_coarse_direct_vcycle_and_pcg(gpu, oracle, n, ml, nc):
    A = P.poisson3d(n)
    dA = gpu.CsrMatrix.from_arrays(*A)
    H = gpu.Hierarchy(dA, kind=L.AMG_SA, max_level=ml)
    assert H.levels == ml and H.A(ml).info()[0] == nc
    Ho = oracle.amg_setup(A, kind=0, max_level=ml)
    r = np.random.default_rng(1).uniform(-1, 1, A[0].size - 1)
    opts = gpu.amg_options(omega=2.0 / 3.0, coarse=L.COARSE_DIRECT)
    z = H.cycle(gpu.vec(r), options=opts).cpu().numpy()
    zo = Ho.vcycle(r, omega=2.0 / 3.0, coarse=1)
    # the two inverses round differently; the coarsest operator's condition number
    # (a few hundred here) scales that into the cycle
    assert np.max(np.abs(z - zo)) <= 1e-10 * np.max(np.abs(zo))
    b, _ = P.rhs_from_solution(*A, seed=0)
    x, info = gpu.pcg(dA, gpu.vec(b), M=gpu.Preconditioner.amg(H, opts),
                      control=gpu.iter_control(rel_tol=1e-8, abs_tol=0.0, max_iter=500))
    xo, ito, _ = Ho.pcg(b, omega=2.0 / 3.0, coarse=1, rel_tol=1e-8, abs_tol=0.0, max_iter=500)
    assert info.converged and abs(info.iterations - ito) <= 1, (info.iterations, ito)
    assert np.max(np.abs(x.cpu().numpy() - xo)) <= 1e-7 * np.max(np.abs(xo))
