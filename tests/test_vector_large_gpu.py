"""VECTOR SpMV (W lanes per row, every W) on matrices of 1-1.6 M entries.
Integer-valued matrices and vectors make every summation order exact, so an
indexing slip (lane-strided entries, row ends, rows of up to 4000 entries
between short ones, empty rows) shows as a difference from numpy;
real-valued cases follow the reference's SpMV acceptance bound
(clients/common/utility.cpp:526-544)."""
import numpy as np
import pytest

from linalglib_b200 import _lib as L

pytestmark = pytest.mark.gpu


def _csr_from_lens(lens, n, rng, ints):
    m = lens.size
    rp = np.zeros(m + 1, dtype=np.int64)
    np.cumsum(lens, out=rp[1:])
    nnz = int(rp[-1])
    # sorted distinct columns per row: a random start and strictly increasing gaps
    gaps = rng.integers(1, 4, size=nnz)
    starts = np.repeat(np.arange(m), lens)
    first = np.zeros(nnz, dtype=bool)
    first[rp[:-1][lens > 0]] = True
    gaps[first] = 0
    seg = np.cumsum(gaps)
    seg -= np.repeat(seg[rp[:-1]], lens) if nnz else seg
    base = rng.integers(0, n, size=m)
    ci = (np.repeat(base, lens) + seg) % n
    # keep each row sorted after the wrap-around
    order = np.lexsort((ci, starts))
    ci = ci[order]
    if ints:
        v = rng.integers(-3, 4, size=nnz).astype(np.float64)
    else:
        v = rng.uniform(-1, 1, size=nnz)
    return rp.astype(np.int32), ci.astype(np.int32), v


def _dense_ref(rp, ci, v, x):
    rows = np.repeat(np.arange(rp.size - 1), np.diff(rp))
    y = np.zeros(rp.size - 1)
    np.add.at(y, rows, v * x[ci])
    return y


CASES = {
    # mean 41 (an SA level-1 operator's rows), Poisson lengths, some empty rows
    "mean41": lambda rng: rng.poisson(41, size=40000),
    # mean 143 with a wide spread
    "mean143": lambda rng: rng.integers(0, 290, size=9000),
    # short rows with a long row every 997 rows
    "spiky": lambda rng: np.where(np.arange(150000) % 997 == 5, 4000, rng.poisson(6, size=150000)),
    # rows of ~1000 entries
    "long": lambda rng: rng.integers(900, 1100, size=1100),
}


@pytest.mark.parametrize("case", list(CASES))
@pytest.mark.parametrize("lanes", [2, 4, 8, 16, 32])
def test_vector_exact_on_integers(gpu, case, lanes):
    rng = np.random.default_rng(lanes * 31 + len(case))
    lens = CASES[case](rng).astype(np.int64)
    n = 50000
    lens = np.minimum(lens, n // 4)
    rp, ci, v = _csr_from_lens(lens, n, rng, ints=True)
    assert rp[-1] >= 1 << 20
    x = rng.integers(-4, 5, size=n).astype(np.float64)
    y0 = rng.integers(-4, 5, size=rp.size - 1).astype(np.float64)
    A = gpu.CsrMatrix.from_arrays(rp, ci, v, n=n)
    A.set_algorithm(L.SPMV_VECTOR, lanes)
    y = A.spmv(gpu.vec(x), gpu.vec(y0), alpha=2.0, beta=-1.0).cpu().numpy()
    assert np.array_equal(y, 2.0 * _dense_ref(rp, ci, v, x) - y0)


@pytest.mark.parametrize("lanes", [4, 8, 16])
def test_vector_matches_oracle(gpu, oracle, lanes):
    rng = np.random.default_rng(5 + lanes)
    lens = rng.poisson(41, size=30000).astype(np.int64)
    n = 30000
    rp, ci, v = _csr_from_lens(lens, n, rng, ints=False)
    x = rng.uniform(-1, 1, n)
    A = gpu.CsrMatrix.from_arrays(rp, ci, v, n=n)
    A.set_algorithm(L.SPMV_VECTOR, lanes)
    y = A.spmv(gpu.vec(x)).cpu().numpy()
    yo = oracle.spmv((rp, ci, v, n), x)
    assert np.max(np.abs(y - yo)) <= 1e-9
    # deterministic: a second run is identical
    assert np.array_equal(A.spmv(gpu.vec(x)).cpu().numpy(), y)


def _timeouts(gpu):
    import ctypes as C
    n = C.c_int64()
    L.call("lab_wait_timeouts", C.byref(n), gpu.stream_handle())
    return n.value


@pytest.mark.parametrize("case", ["mean41", "spiky"])
@pytest.mark.parametrize("lanes", [2, 4, 8, 16, 32])
def test_vector_streamed_equals_direct(gpu, case, lanes):
    """The streamed VECTOR schedule (the matrix moved through shared memory by bulk
    copies, one producer warp) sums each row exactly as the direct-load kernel
    does, so the results are bit-identical."""
    rng = np.random.default_rng(77 + lanes)
    lens = CASES[case](rng).astype(np.int64)
    n = 60000
    rp, ci, v = _csr_from_lens(np.minimum(lens, 800), n, rng, ints=False)
    x = gpu.vec(rng.uniform(-1, 1, n))
    y0 = rng.uniform(-1, 1, rp.size - 1)
    A = gpu.CsrMatrix.from_arrays(rp, ci, v, n=n)
    before = _timeouts(gpu)
    out = {}
    for alg in (L.SPMV_VECTOR, L.SPMV_VECTOR_STREAM):
        A.set_algorithm(alg, lanes)
        out[alg] = A.spmv(x, gpu.vec(y0), alpha=1.5, beta=-0.5).cpu().numpy()
    # the library's tile rule: whole consumer passes (8 warps x 32 / W rows) of about
    # 2048 entries; the matrix streams if its largest tile (+16) fits 4096 entries
    m = rp.size - 1
    avg = rp[-1] / m
    rpp = 8 * 32 // lanes
    rows = min(1024, rpp * max(1, int(2048 / avg / rpp)))
    r0 = np.arange(0, m, rows)
    biggest = int(np.max(rp[np.minimum(r0 + rows, m)] - rp[r0]))
    streams = m >= 8192 and biggest + 16 <= 4096
    assert A.algorithm() == ((L.SPMV_VECTOR_STREAM if streams else L.SPMV_VECTOR), lanes)
    if case == "mean41" and lanes == 8:
        assert streams
    assert np.array_equal(out[L.SPMV_VECTOR].view(np.int64), out[L.SPMV_VECTOR_STREAM].view(np.int64))
    assert _timeouts(gpu) == before


@pytest.mark.parametrize("prec", [L.PREC_FP64, L.PREC_FP32, L.PREC_FP32_BF16])
def test_cycle_streamed_equals_direct(gpu, prec):
    """A V-cycle (FP64, FP32 and FP32 + BF16 values) whose large coarse operators
    and restriction run streamed equals the default cycle (every VECTOR pass
    reading global memory directly), bit for bit."""
    from linalglib_b200 import problems as P
    A = P.poisson3d(64)
    dA = gpu.CsrMatrix.from_arrays(*A)
    H = gpu.Hierarchy(dA)
    r = gpu.vec(np.random.default_rng(1).uniform(-1, 1, A[0].size - 1))
    mats = [H.A(l) for l in range(H.levels + 1)] + [H.R(l) for l in range(H.levels)]
    vec_mats = [(M, M.algorithm()[1]) for M in mats
                if M.algorithm()[0] in (L.SPMV_VECTOR, L.SPMV_VECTOR_HALO)]
    assert any(M.m >= 8192 for M, _ in vec_mats)
    M = gpu.Preconditioner.amg(H, gpu.amg_options(precision=prec))
    z_direct = M.apply(r).cpu().numpy()
    for Mx, w in vec_mats:
        Mx.set_algorithm(L.SPMV_VECTOR_STREAM, w)
    z_stream = M.apply(r).cpu().numpy()
    assert np.array_equal(z_stream.view(np.int64), z_direct.view(np.int64))
    assert _timeouts(gpu) == 0
