"""Triangular path on the CPU: the C restatement (oracle/oracle.c) against the
compiled reference -- ILU(0), IC(0), lower/upper triangular solves and the
ILU(0) / IC(0) / Gauss-Seidel / SOR / SSOR preconditioner applications must agree
bit for bit (host_csrilu0.cpp, host_csric0.cpp, host_csrtrsv.cpp, preconditioner.cpp)."""
import numpy as np
import pytest

from linalglib_b200 import problems as P

CASES = {
    "poisson2d_20": lambda: P.poisson2d(20),
    "laplacian3d_8": lambda: P.graph_laplacian3d(8, seed=1),
    "diffusion27_6": lambda: P.diffusion27(6, seed=2),
}


@pytest.mark.parametrize("name", list(CASES))
@pytest.mark.parametrize("fn", ["csrilu0", "csric0"])
def test_factorizations_oracle_vs_reference(oracle, reference, name, fn):
    A = CASES[name]()
    vo, so, no = getattr(oracle, fn)(A)
    vr, sr, nr = getattr(reference, fn)(A)
    assert np.array_equal(vo.view(np.int64), vr.view(np.int64))
    assert (so, no) == (sr, nr)


@pytest.mark.parametrize("name", list(CASES))
@pytest.mark.parametrize("lower", [True, False])
@pytest.mark.parametrize("unit", [True, False])
def test_trsv_oracle_vs_reference(oracle, reference, name, lower, unit):
    A = CASES[name]()
    b = np.random.default_rng(3).uniform(-1, 1, A[0].size - 1)
    assert np.array_equal(oracle.trsv(A, b, lower, unit), reference.trsv(A, b, lower, unit))


@pytest.mark.parametrize("name", list(CASES))
@pytest.mark.parametrize("kind", [0, 1, 2, 3, 4])
def test_precond_apply_oracle_vs_reference(oracle, reference, name, kind):
    A = CASES[name]()
    r = np.random.default_rng(4).uniform(-1, 1, A[0].size - 1)
    xo = oracle.precond_apply(kind, A, r, omega=1.3)
    xr = reference.precond_apply(kind, A, r, omega=1.3)
    assert np.array_equal(xo, xr)


def test_zero_pivots_reported_like_reference(oracle, reference):
    # a zero on the diagonal of row 3 (numeric zero) and a missing diagonal in
    # row 5 (structural zero): both factorizations substitute 1.0 and report the
    # smallest such column, and ILU(0)'s update loop then starts at position 0
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
         ci[keep], v[keep])
    for fn in ("csrilu0", "csric0"):
        vo, so, no = getattr(oracle, fn)(A)
        vr, sr, nr = getattr(reference, fn)(A)
        assert np.array_equal(vo.view(np.int64), vr.view(np.int64)), fn
        assert (so, no) == (sr, nr), fn


@pytest.mark.parametrize("kind", [0, 1, 2, 3, 4])
def test_precond_cg_oracle_vs_reference(oracle, reference, kind):
    # the whole preconditioned CG (ILU(0) and SSOR converge; IC(0) as the
    # reference applies it, Gauss-Seidel and SOR are not symmetric and stagnate).  The
    # reference's dot products are OpenMP reductions, so the iterates agree to
    # rounding, not bit for bit.
    A = P.poisson2d(24)
    b, _ = P.rhs_from_solution(*A[:3], seed=0)
    xo, io = oracle.precond_cg(kind, A, b, omega=1.3, max_iter=60)
    xr, ir = reference.precond_cg(kind, A, b, omega=1.3, max_iter=60)
    assert io == ir
    tol = 1e-9 if kind in (0, 4) else 1e-6
    assert np.max(np.abs(xo - xr)) <= tol * np.max(np.abs(xr))


@pytest.mark.parametrize("n,per_row,seed", [(2, 2, 1), (300, 6, 2)])
def test_nonsymmetric_patterns_oracle_vs_reference(oracle, reference, n, per_row, seed):
    rng = np.random.default_rng(seed)
    rp, ci, v = [0], [], []
    for i in range(n):
        cols = sorted(set(rng.choice(n, size=min(per_row, n), replace=False).tolist()) | {i})
        vals = rng.uniform(-1, 1, len(cols))
        vals[cols.index(i)] = len(cols) + 1.0
        ci += cols
        v += vals.tolist()
        rp.append(len(ci))
    A = (np.array(rp, np.int32), np.array(ci, np.int32), np.array(v))
    b = rng.uniform(-1, 1, n)
    for kind in range(5):
        assert np.array_equal(oracle.precond_apply(kind, A, b, omega=1.3).view(np.int64),
                              reference.precond_apply(kind, A, b, omega=1.3).view(np.int64))
    for fn in ("csrilu0", "csric0"):
        vo, so, no = getattr(oracle, fn)(A)
        vr, sr, nr = getattr(reference, fn)(A)
        assert np.array_equal(vo.view(np.int64), vr.view(np.int64)) and (so, no) == (sr, nr)
