"""Level-scheduled triangular path on the GPU: lab_csrtrsv, lab_csrilu0 /
lab_csric0 and the ILU(0) / IC(0) / Gauss-Seidel / SOR / SSOR preconditioners are
bit-identical to the oracle (which is pinned bit-exact to the reference's
host_csrtrsv.cpp, host_csrilu0.cpp, host_csric0.cpp and preconditioner.cpp), and
PCG with them behaves as the reference's cg_solver does."""
import numpy as np
import pytest

from linalglib_b200 import problems as P

pytestmark = pytest.mark.gpu

CASES = {
    "poisson2d_20": lambda: P.poisson2d(20),
    "laplacian3d_8": lambda: P.graph_laplacian3d(8, seed=1),
    "diffusion27_6": lambda: P.diffusion27(6, seed=2),
    "poisson3d_24": lambda: P.poisson3d(24),
}


def _bits(a):
    return np.ascontiguousarray(a, dtype=np.float64).view(np.int64)


@pytest.mark.parametrize("name", list(CASES))
@pytest.mark.parametrize("lower", [True, False])
@pytest.mark.parametrize("unit", [True, False])
def test_trsv_bit_exact(gpu, oracle, name, lower, unit):
    A = CASES[name]()
    b = np.random.default_rng(3).uniform(-1, 1, A[0].size - 1)
    x = gpu.CsrMatrix.from_arrays(*A[:3]).trsv(gpu.vec(b), lower=lower, unit_diag=unit)
    assert np.array_equal(_bits(x.cpu().numpy()), _bits(oracle.trsv(A, b, lower, unit)))


@pytest.mark.parametrize("name", list(CASES))
@pytest.mark.parametrize("kind", ["ilu0", "ic0"])
def test_factor_bit_exact(gpu, oracle, name, kind):
    A = CASES[name]()
    dA = gpu.CsrMatrix.from_arrays(*A[:3])
    sz, nz = dA.factor(kind)
    vo, so, no = getattr(oracle, "csr" + kind)(A)
    big = np.iinfo(np.int32).max
    assert (sz, nz) == (-1 if so == big else so, -1 if no == big else no)
    assert np.array_equal(_bits(dA.to_numpy()[2]), _bits(vo))


def test_factor_zero_pivots(gpu, oracle):
    # numeric zero on row 3's diagonal, structural zero (no diagonal) in row 5:
    # the level-parallel and sequential paths must both report the smallest column
    rp, ci, v = P.poisson2d(4)
    v = v.copy()
    for j in range(rp[3], rp[4]):
        if ci[j] == 3:
            v[j] = 0.0
    keep = np.ones(v.size, dtype=bool)
    for j in range(rp[5], rp[6]):
        if ci[j] == 5:
            keep[j] = False
    rows = np.repeat(np.arange(rp.size - 1), np.diff(rp))[keep]
    A = (np.concatenate([[0], np.cumsum(np.bincount(rows, minlength=rp.size - 1))]).astype(np.int32),
         ci[keep].copy(), v[keep].copy())
    for kind in ("ilu0", "ic0"):
        dA = gpu.CsrMatrix.from_arrays(*A)
        sz, nz = dA.factor(kind)
        vo, so, no = getattr(oracle, "csr" + kind)(A)
        big = np.iinfo(np.int32).max
        assert (sz, nz) == (-1 if so == big else so, -1 if no == big else no), kind
        assert np.array_equal(_bits(dA.to_numpy()[2]), _bits(vo)), kind


def _precond(gpu, kind, dA, omega=1.3):
    return [gpu.Preconditioner.ilu0, gpu.Preconditioner.ic0, gpu.Preconditioner.gauss_seidel,
            lambda X: gpu.Preconditioner.sor(X, omega),
            lambda X: gpu.Preconditioner.ssor(X, omega)][kind](dA)


@pytest.mark.parametrize("name", list(CASES))
@pytest.mark.parametrize("kind", [0, 1, 2, 3, 4])
def test_precond_apply_bit_exact(gpu, oracle, name, kind):
    A = CASES[name]()
    dA = gpu.CsrMatrix.from_arrays(*A[:3])
    M = _precond(gpu, kind, dA)
    r = np.random.default_rng(4).uniform(-1, 1, A[0].size - 1)
    z = M.apply(gpu.vec(r)).cpu().numpy()
    assert np.array_equal(_bits(z), _bits(oracle.precond_apply(kind, A, r, omega=1.3)))
    # the preconditioner works on a copy: A itself is unchanged
    assert np.array_equal(_bits(dA.to_numpy()[2]), _bits(A[2]))


@pytest.mark.parametrize("kind,omega,expected", [(0, 1.0, 24), (4, 1.3, 32), (4, 1.0, 26)])
def test_ilu_ssor_pcg_matches_reference(gpu, reference, kind, omega, expected):
    A = P.poisson2d(24)
    b, xt = P.rhs_from_solution(*A[:3], seed=0)
    dA = gpu.CsrMatrix.from_arrays(*A[:3])
    x, info = gpu.pcg(dA, gpu.vec(b), M=_precond(gpu, kind, dA, omega),
                      control=gpu.iter_control(rel_tol=1e-8, abs_tol=0.0, max_iter=1000))
    xr, itr = reference.precond_cg(kind, A, b, omega=omega, rel_tol=1e-8, abs_tol=1e-300)
    assert itr == expected  # the reference's count on this problem
    assert info.converged == 1
    assert abs(info.iterations - itr) <= 1, (info.iterations, itr)
    assert np.max(np.abs(x.cpu().numpy() - xr)) <= 1e-7 * np.max(np.abs(xr))
    assert np.max(np.abs(x.cpu().numpy() - xt)) <= 1e-6


@pytest.mark.parametrize("kind", [1, 2, 3])
def test_nonsymmetric_precond_pcg_like_reference(gpu, reference, kind):
    # The reference's IC(0) factor overwrites only the lower triangle and its
    # upper solve reads the unfactored upper part (host_csric0.cpp:70-115,
    # preconditioner.cpp:512-525); Gauss-Seidel and SOR are one-sided.  None is
    # symmetric, so the reference's CG stagnates with them: the device path must
    # do the same (not converged, the same iterate after 50 iterations).
    A = P.poisson2d(24)
    b, _ = P.rhs_from_solution(*A[:3], seed=0)
    dA = gpu.CsrMatrix.from_arrays(*A[:3])
    M = _precond(gpu, kind, dA)
    x, info = gpu.pcg(dA, gpu.vec(b), M=M,
                      control=gpu.iter_control(rel_tol=1e-8, abs_tol=0.0, max_iter=50))
    xr, itr = reference.precond_cg(kind, A, b, omega=1.3, rel_tol=1e-8, abs_tol=1e-300,
                                   max_iter=50)
    assert itr == 51 and info.converged == 0
    assert np.max(np.abs(x.cpu().numpy() - xr)) <= 1e-6 * np.max(np.abs(xr))


@pytest.mark.parametrize("name", ["poisson3d_24", "diffusion27_6"])
def test_nonsymmetric_preconds_under_gmres(gpu, name):
    # Gauss-Seidel and SOR are one-sided: they work under GMRES (the reference's
    # IC(0), whose upper solve reads the unfactored upper part, does not converge
    # under GMRES either: its application is checked bit for bit above)
    A = CASES[name]()
    b, xt = P.rhs_from_solution(*A[:3], seed=1)
    dA = gpu.CsrMatrix.from_arrays(*A[:3])
    for M in (gpu.Preconditioner.gauss_seidel(dA), gpu.Preconditioner.sor(dA, 1.2)):
        x, info = gpu.gmres(dA, gpu.vec(b), M=M, restart=30,
                            control=gpu.iter_control(rel_tol=1e-10, abs_tol=0.0, max_iter=2000))
        assert info.converged == 1
        assert np.max(np.abs(x.cpu().numpy() - xt)) <= 1e-6 * np.max(np.abs(xt))


def test_trsv_in_place_and_ssor_arg_check(gpu, oracle):
    A = P.poisson3d(12)
    b = np.random.default_rng(7).uniform(-1, 1, A[0].size - 1)
    dA = gpu.CsrMatrix.from_arrays(*A[:3])
    for lower in (True, False):
        xb = gpu.vec(b)
        dA.trsv(xb, lower=lower, unit_diag=False, x=xb)  # b and x the same array
        assert np.array_equal(_bits(xb.cpu().numpy()), _bits(oracle.trsv(A, b, lower, False)))
    from linalglib_b200 import _lib as L
    for bad in (0.0, 2.0, -1.0):
        with pytest.raises(L.LabError):
            gpu.Preconditioner.ssor(dA, bad)


def _random_nonsym(n, per_row, seed):
    """Random nonsymmetric pattern (sorted rows, stored diagonal, a few empty
    off-diagonal rows) with diagonally dominant values."""
    rng = np.random.default_rng(seed)
    rp, ci, v = [0], [], []
    for i in range(n):
        k = 0 if i % 17 == 5 else rng.integers(1, per_row + 1)
        cols = set(rng.choice(n, size=min(k, n), replace=False).tolist()) - {i}
        cols = sorted(cols | {i})
        vals = rng.uniform(-1, 1, len(cols))
        vals[cols.index(i)] = len(cols) + 1.0
        ci += cols
        v += vals.tolist()
        rp.append(len(ci))
    return (np.array(rp, np.int32), np.array(ci, np.int32), np.array(v, np.float64))


@pytest.mark.parametrize("n,per_row,seed", [(1, 1, 0), (2, 2, 1), (300, 6, 2), (2000, 12, 3)])
def test_nonsymmetric_patterns_bit_exact(gpu, oracle, n, per_row, seed):
    # the level analysis reads the dependents of a row through the pattern's
    # transpose: nonsymmetric patterns exercise it
    A = _random_nonsym(n, per_row, seed)
    b = np.random.default_rng(seed + 10).uniform(-1, 1, n)
    dA = gpu.CsrMatrix.from_arrays(*A)
    for lower in (True, False):
        for unit in (True, False):
            x = dA.trsv(gpu.vec(b), lower=lower, unit_diag=unit)
            assert np.array_equal(_bits(x.cpu().numpy()), _bits(oracle.trsv(A, b, lower, unit)))
    for kind in (0, 1, 2, 3, 4):
        z = _precond(gpu, kind, dA).apply(gpu.vec(b)).cpu().numpy()
        assert np.array_equal(_bits(z), _bits(oracle.precond_apply(kind, A, b, omega=1.3))), kind


@pytest.mark.parametrize("lower", [True, False])
def test_trsv_bounded_wait_reports_timeout(gpu, oracle, lower):
    """The solves poll for their dependencies with a bounded wait.  A held row
    (its value never written) makes every row that depends on it run out of its
    wait: the launch must return and the call report LAB_TIMEOUT, and the same
    matrix must solve bit-exactly again once the hold is lifted."""
    import ctypes as C
    from linalglib_b200 import _lib as L
    A = P.poisson3d(24)
    m = A[0].size - 1
    b = np.random.default_rng(4).uniform(-1, 1, m)
    dA = gpu.CsrMatrix.from_arrays(*A[:3])
    held = 0 if lower else m - 1  # the first row solved; every other row depends on it
    L.call("lab_csrtrsv_wait_control", dA.h, 1 << 12, held, gpu.stream_handle())
    bx, x = gpu.vec(b), gpu.vec(np.zeros(m))
    st = L.lib().lab_csrtrsv(dA.h, int(lower), 0, gpu.ptr(bx), gpu.ptr(x), gpu.stream_handle())
    assert st == L.LAB_TIMEOUT, L.lib().lab_last_error().decode()
    assert "wait" in L.lib().lab_last_error().decode()
    L.call("lab_csrtrsv_wait_control", dA.h, 0, -1, gpu.stream_handle())
    x = dA.trsv(gpu.vec(b), lower=lower)
    assert np.array_equal(_bits(x.cpu().numpy()), _bits(oracle.trsv(A, b, lower, False)))


MEMBER_CASES = {
    "poisson2d_20": lambda: P.poisson2d(20),
    "diffusion27_6": lambda: P.diffusion27(6, seed=2),
    "nonsym_18": lambda: _nonsym(18),
}


def _nonsym(n):
    rp, ci, v = P.poisson2d(n)
    v = v.copy()
    rows = np.repeat(np.arange(rp.size - 1), np.diff(rp))
    v[ci == rows + 1] *= 0.37
    v[ci == rows - n] *= 1.9
    return rp, ci, v


@pytest.mark.parametrize("name", list(MEMBER_CASES))
def test_triangle_copies_match_reference(gpu, reference, name):
    """copy_lower_triangular_from / copy_upper_triangular_from
    (csr_matrix.cpp:170-225): same pattern, same values."""
    from helpers import csr_diff, csr_equal
    A = MEMBER_CASES[name]()
    dA = gpu.CsrMatrix.from_arrays(*A)
    for upper in (False, True):
        g = dA.triangle(upper=upper).to_numpy()
        r = reference.triangle(A, upper=upper)
        assert csr_equal(g, r), csr_diff(g, r)


@pytest.mark.parametrize("name", list(MEMBER_CASES))
def test_diagonal_scalings_match_reference(gpu, reference, name):
    """scale_diagonal_by and scale_by_inverse_diagonal (host_scale.cpp:34-69)."""
    A = MEMBER_CASES[name]()
    dA = gpu.CsrMatrix.from_arrays(*A)
    dA.scale_diagonal(-2.75)
    assert np.array_equal(_bits(dA.to_numpy()[2]), _bits(reference.scale_diagonal(A, -2.75)))
    dB = gpu.CsrMatrix.from_arrays(*A)
    dB.scale_by_inverse_diagonal()
    assert np.array_equal(_bits(dB.to_numpy()[2]), _bits(reference.scale_by_inverse_diagonal(A)))
    # the scaled matrix's cached diagonal is rebuilt (the next Jacobi sees new values)
    assert np.array_equal(dB.diagonal().cpu().numpy(),
                          [dB.to_numpy()[2][j] for j in
                           [next(k for k in range(A[0][i], A[0][i + 1]) if A[1][k] == i)
                            for i in range(A[0].size - 1)]])
