"""AMG setup on the GPU vs the oracle: every integer output and every value of
P, R and A_c must be bit-identical (the reference's own acceptance for SpGEMM is
exact equality, clients/common/utility.cpp:478-524; for strength / aggregation
there is no tolerance to give).
"""
import numpy as np
import pytest
import torch

from linalglib_b200 import _lib as L
from linalglib_b200 import problems as P

from helpers import bits_equal, csr_diff, csr_equal

pytestmark = pytest.mark.gpu

PROBLEMS = {
    "poisson2d_33": lambda: P.poisson2d(33),
    "poisson2d_64x40": lambda: P.poisson2d(64, 40),
    "poisson3d_16": lambda: P.poisson3d(16),
    "laplacian3d_12": lambda: P.graph_laplacian3d(12, seed=3),
    "diffusion27_8": lambda: P.diffusion27(8, seed=1),
}


def _A(gpu, A):
    return gpu.CsrMatrix.from_arrays(*A[:3], n=(A[3] if len(A) > 3 else None))


@pytest.mark.parametrize("name", list(PROBLEMS))
def test_strength_pmis_prolongation_level0(gpu, oracle, name):
    A = PROBLEMS[name]()
    dA = _A(gpu, A)
    m, nnz = A[0].size - 1, A[2].size
    for eps in (0.08, 0.001, 0.3):
        conn = torch.zeros(nnz, dtype=torch.int32, device="cuda")
        L.call("lab_strength", dA.h, eps, gpu.ptr(conn), gpu.stream_handle())
        co = oracle.strength(A, eps)
        assert np.array_equal(conn.cpu().numpy(), co)
    eps = 0.08
    co = oracle.strength(A, eps)
    conn = torch.as_tensor(co, device="cuda")
    agg = torch.zeros(m, dtype=torch.int64, device="cuda")
    import ctypes
    rounds = ctypes.c_int()
    L.call("lab_pmis_aggregate", dA.h, gpu.ptr(conn), gpu.ptr(agg), ctypes.byref(rounds),
           gpu.stream_handle())
    ao, ro = oracle.pmis(A, co)
    assert np.array_equal(agg.cpu().numpy(), ao)
    assert rounds.value == ro
    h = ctypes.c_void_p()
    L.call("lab_sa_prolongation", dA.h, gpu.ptr(conn), gpu.ptr(agg), 2.0 / 3.0, ctypes.byref(h),
           gpu.stream_handle())
    Pg = gpu.CsrMatrix(h).to_numpy()
    Po = oracle.sa_prolongation(A, co, ao)
    assert csr_equal(Pg, Po), csr_diff(Pg, Po)
    h = ctypes.c_void_p()
    L.call("lab_ua_prolongation", dA.h, gpu.ptr(agg), ctypes.byref(h), gpu.stream_handle())
    Pu = gpu.CsrMatrix(h).to_numpy()
    assert csr_equal(Pu, oracle.ua_prolongation(A, ao))


@pytest.mark.parametrize("name", list(PROBLEMS))
def test_transpose_spgemm_spgeam(gpu, oracle, name):
    A = PROBLEMS[name]()
    m = A[0].size - 1
    dA = _A(gpu, A)
    T = dA.transpose().to_numpy()
    assert csr_equal(T, oracle.transpose((*A[:3], m))), "transpose"
    C = dA.spgemm(dA).to_numpy()
    assert csr_equal(C, oracle.spgemm((*A[:3], m), (*A[:3], m))), "A*A"
    # rectangular: A * P with the SA prolongation
    co = oracle.strength(A, 0.08)
    ao, _ = oracle.pmis(A, co)
    Po = oracle.sa_prolongation(A, co, ao)
    dP = gpu.CsrMatrix.from_arrays(*Po[:3], n=Po[3])
    AP = dA.spgemm(dP).to_numpy()
    APo = oracle.spgemm((*A[:3], m), Po)
    assert csr_equal(AP, APo), csr_diff(AP, APo)
    R = dP.transpose()
    RAP = R.spgemm(gpu.CsrMatrix.from_arrays(*APo[:3], n=APo[3])).to_numpy()
    assert csr_equal(RAP, oracle.spgemm(oracle.transpose(Po), APo))
    G = dA.spgeam(1.5, -0.25, gpu.CsrMatrix.from_arrays(*T[:3], n=T[3])).to_numpy()
    assert csr_equal(G, oracle.spgeam(1.5, (*A[:3], m), -0.25, T))


def test_spgemm_long_rows(gpu, oracle):
    """Rows past the warp (256) and CTA (4096) item tiers take the larger kernels."""
    rng = np.random.default_rng(4)
    m, n = 300, 5000
    lens = np.where(np.arange(m) % 50 == 0, 2500, rng.integers(1, 30, size=m))
    rp = np.zeros(m + 1, np.int32)
    np.cumsum(lens, out=rp[1:])
    ci = np.concatenate([np.sort(rng.choice(n, size=k, replace=False)) for k in lens]).astype(np.int32)
    v = rng.integers(-3, 4, size=rp[-1]).astype(np.float64)  # exact sums
    B = (rp, ci, v, n)
    rpb = np.arange(0, 3 * n + 1, 3, dtype=np.int32)
    cib = rng.integers(0, 700, size=3 * n).astype(np.int32)
    cib = np.sort(cib.reshape(n, 3), axis=1)
    ok = np.all(np.diff(cib, axis=1) > 0, axis=1)
    cib[~ok] = np.array([0, 1, 2])
    Bm = (rpb, cib.reshape(-1), rng.uniform(-1, 1, 3 * n), 700)
    C = gpu.CsrMatrix.from_arrays(*B[:3], n=n).spgemm(gpu.CsrMatrix.from_arrays(*Bm[:3], n=700))
    assert csr_equal(C.to_numpy(), oracle.spgemm(B, Bm))
    # many distinct columns per row: the hash table overflows into the sort tier
    cib2 = np.sort(rng.choice(6000, size=(n, 3)), axis=1)
    ok2 = np.all(np.diff(cib2, axis=1) > 0, axis=1)
    cib2[~ok2] = np.array([0, 1, 2])
    Bm2 = (rpb, cib2.reshape(-1).astype(np.int32), rng.uniform(-1, 1, 3 * n), 6000)
    C2 = gpu.CsrMatrix.from_arrays(*B[:3], n=n).spgemm(gpu.CsrMatrix.from_arrays(*Bm2[:3], n=6000))
    assert csr_equal(C2.to_numpy(), oracle.spgemm(B, Bm2))


@pytest.mark.parametrize("kind", [L.AMG_SA, L.AMG_UA])
@pytest.mark.parametrize("name", list(PROBLEMS))
def test_hierarchy_bitexact(gpu, oracle, kind, name):
    A = PROBLEMS[name]()
    H = gpu.Hierarchy(_A(gpu, A), kind=kind, max_level=20)
    Ho = oracle.amg_setup(A, kind=kind, max_level=20)
    assert H.levels == Ho.levels
    for l in range(H.levels + 1):
        a, ao = H.A(l).to_numpy(), Ho.A(l)
        assert csr_equal(a, ao), f"A{l}: {csr_diff(a, ao)}"
        if l < H.levels:
            p, po = H.P(l).to_numpy(), Ho.P(l)
            assert csr_equal(p, po), f"P{l}: {csr_diff(p, po)}"
            r, ro = H.R(l).to_numpy(), Ho.R(l)
            assert csr_equal(r, ro), f"R{l}: {csr_diff(r, ro)}"


@pytest.mark.parametrize("max_level", [0, 1, 2])
def test_hierarchy_max_level(gpu, oracle, max_level):
    A = P.poisson2d(20)
    H = gpu.Hierarchy(_A(gpu, A), kind=L.AMG_SA, max_level=max_level)
    Ho = oracle.amg_setup(A, kind=0, max_level=max_level)
    assert H.levels == Ho.levels == max_level
    assert csr_equal(H.A(max_level).to_numpy(), Ho.A(max_level))


@pytest.mark.parametrize("name", ["poisson2d_33", "poisson3d_16", "laplacian3d_12"])
def test_rs_pieces_and_hierarchy(gpu, oracle, name):
    import ctypes
    A = PROBLEMS[name]()
    dA = _A(gpu, A)
    nnz = A[2].size
    conn = torch.zeros(nnz, dtype=torch.int32, device="cuda")
    h = ctypes.c_void_p()
    L.call("lab_classical_strength", dA.h, 0.2, gpu.ptr(conn), ctypes.byref(h), gpu.stream_handle())
    S = gpu.CsrMatrix(h)
    co, So = oracle.classical_strength(A, 0.2)
    assert np.array_equal(conn.cpu().numpy(), co)
    assert csr_equal(S.to_numpy(), So)
    cf = torch.zeros(A[0].size - 1, dtype=torch.int32, device="cuda")
    L.call("lab_cfpoints", S.h, gpu.ptr(cf), gpu.stream_handle())
    cfo = oracle.cfpoints(So)
    assert np.array_equal(cf.cpu().numpy().astype(np.uint32), cfo)
    h = ctypes.c_void_p()
    L.call("lab_direct_interpolation", dA.h, S.h, gpu.ptr(cf), ctypes.byref(h), gpu.stream_handle())
    assert csr_equal(gpu.CsrMatrix(h).to_numpy(), oracle.direct_interpolation(A, So, cfo))
    H = gpu.Hierarchy(dA, kind=L.AMG_RS, max_level=20)
    Ho = oracle.amg_setup(A, kind=2, max_level=20)
    assert H.levels == Ho.levels
    for l in range(H.levels + 1):
        assert csr_equal(H.A(l).to_numpy(), Ho.A(l)), f"A{l}"


def test_hierarchy_matches_reference(gpu, reference):
    """Direct check against the reference library itself (not the restatement)."""
    A = P.poisson2d(48)
    H = gpu.Hierarchy(_A(gpu, A), kind=L.AMG_SA)
    Hr = reference.amg_setup(A, kind=0)
    assert H.levels == Hr.levels
    for l in range(H.levels + 1):
        assert csr_equal(H.A(l).to_numpy(), Hr.A(l))
