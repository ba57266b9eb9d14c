"""CPU tests: the C restatement (oracle.c) pinned against the reference itself
(compiled from its own sources into oracle/_ref) and against the committed golden
fixtures the reference produced (tests/golden/make_golden.py).
"""
import os

import numpy as np
import pytest

from linalglib_b200 import problems as P

from helpers import bits_equal, csr_diff, csr_equal

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")

SMALL = {
    "poisson2d_33": lambda: P.poisson2d(33),
    "poisson2d_50x20": lambda: P.poisson2d(50, 20),
    "poisson3d_12": lambda: P.poisson3d(12),
    "laplacian3d_10": lambda: P.graph_laplacian3d(10, seed=4),
    "diffusion27_6": lambda: P.diffusion27(6, seed=2),
}


@pytest.mark.parametrize("name", list(SMALL))
@pytest.mark.parametrize("kind", [0, 1, 2])
def test_hierarchy_oracle_vs_reference(oracle, reference, name, kind):
    A = SMALL[name]()
    ho = oracle.amg_setup(A, kind=kind)
    hr = reference.amg_setup(A, kind=kind)
    assert ho.levels == hr.levels
    for l in range(ho.levels + 1):
        assert csr_equal(ho.A(l), hr.A(l)), f"A{l}: {csr_diff(ho.A(l), hr.A(l))}"
        if l < ho.levels:
            assert csr_equal(ho.P(l), hr.P(l)), f"P{l}"
            assert csr_equal(ho.R(l), hr.R(l)), f"R{l}"


@pytest.mark.parametrize("name", list(SMALL))
def test_pieces_oracle_vs_reference(oracle, reference, name):
    A = SMALL[name]()
    m = A[0].size - 1
    for eps in (0.08, 0.001):
        assert np.array_equal(oracle.strength(A, eps), reference.strength(A, eps))
    conn = oracle.strength(A, 0.08)
    agg, _ = oracle.pmis(A, conn)
    assert np.array_equal(agg, reference.pmis(A, conn))
    co, So = oracle.classical_strength(A)
    cr, Sr = reference.classical_strength(A)
    assert np.array_equal(co, cr) and csr_equal(So, Sr)
    assert np.array_equal(oracle.cfpoints(So), reference.cfpoints(Sr))
    Am = (*A[:3], m)
    assert csr_equal(oracle.transpose(Am), reference.transpose(Am))
    assert csr_equal(oracle.spgemm(Am, Am), reference.spgemm(Am, Am))
    T = oracle.transpose(Am)
    assert csr_equal(oracle.spgeam(0.5, Am, -2.0, T), reference.spgeam(0.5, Am, -2.0, T))
    x = np.random.default_rng(0).uniform(-1, 1, m)
    y0 = np.random.default_rng(1).uniform(-1, 1, m)
    for a, b in ((1.0, 0.0), (1.0, 1.0), (2.0, -0.5)):
        assert bits_equal(oracle.spmv(Am, x, a, b, y0), reference.spmv(Am, x, a, b, y0))
    assert bits_equal(oracle.residual(Am, x, y0), reference.residual(Am, x, y0))
    s = np.random.default_rng(3).integers(0, 3, size=m)
    assert np.array_equal(oracle.exclusive_scan(s), reference.exclusive_scan(s))


@pytest.mark.parametrize("name", ["poisson2d_33", "poisson3d_12", "laplacian3d_10"])
@pytest.mark.parametrize("kind", [0, 1])
def test_pcg_oracle_vs_reference(oracle, reference, name, kind):
    """Same iteration count; solutions agree to the reduction-order noise
    (the reference's dot products are OpenMP reductions)."""
    A = SMALL[name]()
    b, xt = P.rhs_from_solution(*A[:3], seed=0)
    xo, ito, rel = oracle.amg_setup(A, kind).pcg(b, rel_tol=1e-8, abs_tol=0.0)
    xr, itr = reference.amg_setup(A, kind).pcg(b, rel_tol=1e-8, abs_tol=1e-300)
    assert ito == itr
    assert np.max(np.abs(xo - xr)) <= 1e-9 * np.max(np.abs(xr))
    assert rel <= 1e-8


def test_vcycle_oracle_vs_reference(oracle, reference):
    A = P.poisson2d(40)
    r = np.random.default_rng(5).uniform(-1, 1, 1600)
    zo = oracle.amg_setup(A).vcycle(r)
    zr = reference.amg_setup(A, 0).vcycle(r)
    assert bits_equal(zo, zr)


def test_amg_solve_oracle_vs_reference(oracle, reference):
    A = P.poisson2d(40)
    b, _ = P.rhs_from_solution(*A[:3], seed=1)
    xo, ito = oracle.amg_setup(A).amg_solve(b, rel_tol=1e-8, abs_tol=0.0)
    xr, itr = reference.amg_setup(A, 0).amg_solve(b, rel_tol=1e-8, abs_tol=1e-300)
    assert ito == itr
    assert np.max(np.abs(xo - xr)) <= 1e-12 * np.max(np.abs(xr))


@pytest.mark.parametrize("jacobi", [False, True])
def test_cg_oracle_vs_reference(oracle, reference, jacobi):
    A = P.poisson2d(20)
    b, _ = P.rhs_from_solution(*A[:3], seed=2)
    xo, ito = oracle.cg(A, b, jacobi=jacobi, rel_tol=1e-8, abs_tol=0.0, max_iter=200)
    xr, itr = reference.cg(A, b, jacobi=jacobi, rel_tol=1e-8, abs_tol=1e-300, max_iter=200)
    assert ito == itr
    assert np.max(np.abs(xo - xr)) <= 1e-9 * np.max(np.abs(xr))


# ------------------------------------------------------------------ golden fixtures
def _golden_files():
    if not os.path.isdir(GOLDEN):
        return []
    return sorted(f for f in os.listdir(GOLDEN) if f.endswith(".npz"))


@pytest.mark.parametrize("fname", _golden_files())
def test_oracle_matches_golden(oracle, fname):
    """The fixtures were produced by the reference; the oracle must reproduce them."""
    from golden.make_golden import GOLDEN_CASES, build_problem
    g = np.load(os.path.join(GOLDEN, fname))
    case = GOLDEN_CASES[fname[:-4]]
    A = build_problem(case)
    assert np.array_equal(g["A_rp"], A[0]) and np.array_equal(g["A_ci"], A[1])
    h = oracle.amg_setup(A, kind=case["kind"])
    assert h.levels == int(g["levels"])
    for l in range(h.levels + 1):
        a = h.A(l)
        assert np.array_equal(a[0], g[f"A{l}_rp"]) and np.array_equal(a[1], g[f"A{l}_ci"])
        assert bits_equal(a[2], g[f"A{l}_v"]), f"A{l} values"
        if l < h.levels:
            p = h.P(l)
            assert np.array_equal(p[1], g[f"P{l}_ci"]) and bits_equal(p[2], g[f"P{l}_v"])
    if "conn0" in g:
        assert np.array_equal(oracle.strength(A, case.get("eps", 0.08)), g["conn0"])
        agg, _ = oracle.pmis(A, g["conn0"])
        assert np.array_equal(agg, g["agg0"])
    if "pcg_x" in g:
        x, it, _ = h.pcg(g["b"], rel_tol=float(g["rtol"]), abs_tol=0.0)
        assert it == int(g["pcg_iters"])
        assert np.max(np.abs(x - g["pcg_x"])) <= 1e-9 * np.max(np.abs(g["pcg_x"]))


@pytest.mark.parametrize("name", ["poisson2d_33", "diffusion27_7", "nonsym"])
def test_multicolour_colouring_is_proper(oracle, name):
    """The colouring behind the multicolour smoothers: rows of one colour are never
    coupled (in A or A^T), and every colour class is non-empty."""
    from linalglib_b200 import problems as P
    if name == "poisson2d_33":
        A = P.poisson2d(33)
    elif name == "diffusion27_7":
        A = P.diffusion27(7, seed=1)
    else:
        rp, ci, v = P.poisson2d(17)
        rows = np.repeat(np.arange(rp.size - 1), np.diff(rp))
        keep = ~(ci == rows - 17)  # drop one lower neighbour: a non-symmetric pattern
        rows = rows[keep]
        rp = np.concatenate([[0], np.cumsum(np.bincount(rows, minlength=rp.size - 1))]).astype(np.int32)
        A = (rp, ci[keep], v[keep])
    col, nc = oracle.mc_colouring(A)
    rp, ci = A[0], A[1]
    rows = np.repeat(np.arange(rp.size - 1), np.diff(rp))
    off = ci != rows
    assert np.all(col >= 0) and np.all(col < nc)
    assert not np.any(col[rows[off]] == col[ci[off]])
    assert np.array_equal(np.unique(col), np.arange(nc))


@pytest.mark.parametrize("name", ["poisson2d_33", "poisson3d_12"])
@pytest.mark.parametrize("ref_smoother,code,omega", [(1, 2, 1.0), (3, 2, 0.5), (4, 3, 0.5)])
def test_multicolour_stationary_amg_close_to_reference(oracle, reference, name, ref_smoother,
                                                       code, omega):
    """The multicolour GS / SOR / SSOR restatement against the reference's
    lexicographic sweeps in stationary AMG (amg.cpp:516-571): the orderings differ,
    the cycle counts to 1e-8 agree within one."""
    A = SMALL[name]()
    b, _ = P.rhs_from_solution(*A[:3], seed=0)
    xo, ito = oracle.amg_setup(A).amg_solve(b, smoother=code, omega=omega, coarse=0,
                                            rel_tol=1e-8, abs_tol=0.0, max_cycle=300)
    xr, itr = reference.amg_setup(A, kind=0).amg_solve(b, smoother=ref_smoother, rel_tol=1e-8,
                                                       abs_tol=1e-300, max_cycle=300)
    assert itr <= 300 and abs(ito - itr) <= 1, (ito, itr)
    assert np.max(np.abs(xo - xr)) <= 2e-6 * np.max(np.abs(xr))
