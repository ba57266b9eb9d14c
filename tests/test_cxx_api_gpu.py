"""The C++ API as a reference user would call it: the programs in tests/cxx/ are
compiled against include/ with g++ and linked with liblinalg_b200.so, then run
on the GPU and checked against the oracle."""
import os
import subprocess

import numpy as np
import pytest

from linalglib_b200 import problems as P

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIBDIR = os.path.join(ROOT, "linalglib_b200")


def _compile(tmp_path_factory, name):
    exe = str(tmp_path_factory.mktemp("cxx") / name)
    subprocess.run(["/usr/bin/g++", "-O2", "-std=c++17", "-I", os.path.join(ROOT, "include"),
                    os.path.join(ROOT, "tests", "cxx", name + ".cpp"), "-o", exe, "-L", LIBDIR,
                    "-llinalg_b200", f"-Wl,-rpath,{LIBDIR}"], check=True)
    return exe


@pytest.fixture(scope="module")
def example(tmp_path_factory):
    return _compile(tmp_path_factory, "pcg_amg_example")


def test_cxx_example_matches_oracle(gpu, oracle, example):
    n = 96
    out = subprocess.run([example, str(n)], capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stdout + out.stderr
    levels, cycles, iters, conv, err1, err2, rel, nnz_total = out.stdout.split()
    A = P.poisson2d(n)
    h = oracle.amg_setup(A)
    assert int(levels) == h.levels
    assert int(nnz_total) == sum(h.A(l)[2].size for l in range(h.levels + 1))
    b = P.csr_matvec(*A[:3], np.ones(n * n))
    _, it_o, _ = h.pcg(b, rel_tol=1e-8, abs_tol=0.0, coarse=1)
    assert abs(int(iters) - it_o) <= 1
    _, cyc_o = h.amg_solve(b, rel_tol=1e-8, abs_tol=0.0, max_cycle=300, coarse=1)
    assert abs(int(cycles) - cyc_o) <= 1
    assert int(conv) == 1 and float(rel) <= 1e-8


def test_cxx_triangular_preconditioners(gpu, oracle, reference, tmp_path_factory):
    exe = _compile(tmp_path_factory, "tri_precond_example")
    n = 24
    out = subprocess.run([exe, str(n)], capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stdout + out.stderr
    lines = out.stdout.split("\n")
    iters, conv, gs_cycles, sor_cycles, rel, sz, nz, ssor_iters = lines[0].split()
    A = P.poisson2d(n)
    m, nnz = n * n, A[2].size
    vals = np.array([float.fromhex(t) for t in lines[1:1 + nnz]])
    y = np.array([float.fromhex(t) for t in lines[1 + nnz:1 + nnz + m]])
    vo, so, no = oracle.csrilu0(A)
    assert np.array_equal(vals.view(np.int64), vo.view(np.int64))
    assert (int(sz), int(nz)) == (-1, -1) and (so, no) == (np.iinfo(np.int32).max,) * 2
    y_o = oracle.trsv((A[0], A[1], vo), np.ones(m), True, True)
    assert np.array_equal(y.view(np.int64), y_o.view(np.int64))
    b = P.csr_matvec(*A[:3], np.ones(m))
    _, itr = reference.precond_cg(0, A, b, rel_tol=1e-8, abs_tol=1e-300, max_iter=1000)
    assert int(conv) == 1 and abs(int(iters) - itr) <= 1, (iters, itr)
    _, its = reference.precond_cg(4, A, b, omega=1.3, rel_tol=1e-8, abs_tol=1e-300, max_iter=1000)
    assert abs(int(ssor_iters) - its) <= 1, (ssor_iters, its)
    # GMRES stops on the preconditioned 2-norm residual (1e-10 relative); the
    # printed figure is the true inf-norm residual
    assert float(rel) <= 1e-8


def test_cxx_matrix_members_and_mtx(gpu, reference, tmp_path_factory, tmp_path):
    """read_mtx, the triangle copies, diagonal scalings, IC(0) / ILU(0) (members
    and descriptor form), write_mtx and the triangular-solve members, called as a
    reference client calls them; every file written must be byte-identical to the
    reference's write_mtx of the reference's own result, and the solves bitwise."""
    from linalglib_b200 import _lib as L
    exe = _compile(tmp_path_factory, "matrix_members_example")
    n = 14
    rp, ci, v = P.poisson2d(n)
    v = v.copy()
    rows = np.repeat(np.arange(rp.size - 1), np.diff(rp))
    v[ci == rows + 1] *= 0.625
    v[ci == rows] += np.linspace(0.0, 1.0, rp.size - 1)
    src = tmp_path / "in.mtx"
    L.mtx_write(src, rp, ci, v)
    out = subprocess.run([exe, str(src), str(tmp_path)], capture_output=True, text=True,
                         timeout=300)
    assert out.returncode == 0, out.stdout + out.stderr
    A = reference.read_mtx(src)
    m = A[0].size - 1

    def same(name, R):
        reference.write_mtx(tmp_path / ("ref_" + name), R)
        assert (tmp_path / name).read_bytes() == (tmp_path / ("ref_" + name)).read_bytes(), name

    same("lower.mtx", reference.triangle(A, upper=False))
    same("upper.mtx", reference.triangle(A, upper=True))
    same("diag.mtx", (A[0], A[1], reference.scale_diagonal(A, 2.5), A[3]))
    same("invdiag.mtx", (A[0], A[1], reference.scale_by_inverse_diagonal(A), A[3]))
    for name, fn in (("ic0", reference.csric0), ("ilu0", reference.csrilu0)):
        R = (A[0], A[1], fn(A)[0], A[3])
        same(name + ".mtx", R)
        same(name + "_descr.mtx", R)
    xs = np.array([float.fromhex(t) for t in out.stdout.split()])
    xl, xu = xs[:m], xs[m:]
    assert np.array_equal(xl.view(np.int64), reference.trsv(A, np.ones(m), True, False).view(np.int64))
    assert np.array_equal(xu.view(np.int64), reference.trsv(A, np.ones(m), False, False).view(np.int64))


def _random_csr(rng, m, n, per_row):
    """Sorted distinct columns, per_row per row on average, values U[-1, 1]."""
    rows = np.repeat(np.arange(m), rng.integers(1, 2 * per_row, size=m))
    key = np.unique(rows.astype(np.int64) * n + rng.integers(0, n, size=rows.size))
    rp = np.zeros(m + 1, dtype=np.int64)
    np.add.at(rp, key // n + 1, 1)
    return (np.cumsum(rp).astype(np.int32), (key % n).astype(np.int32),
            rng.uniform(-1, 1, key.size), n)


def _write_mtx_exact(path, A):
    rp, ci, v, n = A
    m = rp.size - 1
    rows = np.repeat(np.arange(m), np.diff(rp))
    with open(path, "w") as f:
        f.write("%%MatrixMarket matrix coordinate real general\n")
        f.write(f"{m} {n} {ci.size}\n")
        for r, c, x in zip(rows, ci, v):
            f.write(f"{r + 1} {c + 1} {float(x)!r}\n")


@pytest.fixture(scope="module")
def csrgemm_exe(tmp_path_factory):
    return _compile(tmp_path_factory, "csrgemm_example")


@pytest.mark.parametrize("alpha, beta", [(1.0, 0.0), (0.3, 0.0), (-1.7, 0.45)])
def test_cxx_csrgemm_matches_reference(gpu, reference, csrgemm_exe, tmp_path, alpha, beta):
    """C = alpha A B (+ beta D) through csrgemm_nnz / csrgemm_solve: bit-identical to
    the reference's csrgemm (alpha applied to A's values before the products); the
    beta D term, which the reference's host path does not run, equals its SpGEAM of
    the product and D."""
    from helpers import csr_diff, csr_equal
    rng = np.random.default_rng(17)
    A = _random_csr(rng, 400, 300, 6)
    B = _random_csr(rng, 300, 250, 5)
    D = _random_csr(rng, 400, 250, 4)
    paths = []
    for name, M in (("A", A), ("B", B), ("D", D)):
        paths.append(str(tmp_path / f"{name}.mtx"))
        _write_mtx_exact(paths[-1], M)
    out = subprocess.run([csrgemm_exe, *paths, repr(alpha), repr(beta)], capture_output=True,
                         text=True, timeout=120)
    assert out.returncode == 0, out.stdout + out.stderr
    t = out.stdout.split()
    m, n, nnz = int(t[0]), int(t[1]), int(t[2])
    rp = np.array(t[3:4 + m], dtype=np.int32)
    ci = np.array(t[4 + m:4 + m + nnz], dtype=np.int32)
    v = np.array([float.fromhex(x) for x in t[4 + m + nnz:4 + m + 2 * nnz]])
    ours = (rp, ci, v, n)
    ref = reference.csrgemm(alpha, A, B)
    if beta != 0.0:
        ref = reference.spgeam(1.0, ref, beta, D)
    assert csr_equal(ours, ref), csr_diff(ours, ref)
    if alpha != 1.0:
        # the scaled-after form would differ: the reference rounds (alpha a) b
        scaled_after = reference.spgeam(alpha, reference.spgemm(A, B), 0.0,
                                        reference.spgemm(A, B))
        assert not np.array_equal(scaled_after[2], reference.csrgemm(alpha, A, B)[2])
