"""Hierarchy (de)serialisation: a hierarchy written to a file and loaded back is
bit-identical on every level, gives the same V-cycle and PCG solve, and damaged
or foreign files are refused with LAB_BAD_ARG instead of being half-loaded."""
import numpy as np
import pytest

from linalglib_b200 import _lib as L
from linalglib_b200 import problems as P

from helpers import csr_diff, csr_equal

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("kind,make", [(L.AMG_SA, lambda: P.poisson3d(16)),
                                       (L.AMG_UA, lambda: P.graph_laplacian3d(12, seed=3)),
                                       (L.AMG_RS, lambda: P.poisson2d(24))])
def test_save_load_roundtrip_bit_exact(gpu, tmp_path, kind, make):
    A = make()
    dA = gpu.CsrMatrix.from_arrays(*A)
    H = gpu.Hierarchy(dA, kind=kind)
    path = tmp_path / "h.bin"
    H.save(path)
    G = gpu.Hierarchy.load(path)
    assert G.levels == H.levels
    for l in range(H.levels + 1):
        pairs = [(H.A(l), G.A(l))]
        if l < H.levels:
            pairs += [(H.P(l), G.P(l)), (H.R(l), G.R(l))]
        for X, Y in pairs:
            x, y = X.to_numpy(), Y.to_numpy()
            assert csr_equal(x, y), (l, csr_diff(x, y))
    # (RS levels can hold the reference's 0/0 NaN, rsamg.cpp:838-839, so a cycle may
    # be all NaN: then both must be)
    r = gpu.vec(np.random.default_rng(0).uniform(-1, 1, A[0].size - 1))
    assert np.array_equal(H.cycle(r).cpu().numpy(), G.cycle(r).cpu().numpy(), equal_nan=True)
    b = gpu.vec(P.rhs_from_solution(*A, seed=1)[0])
    ctl = gpu.iter_control(rel_tol=1e-8, abs_tol=0.0)
    x1, i1 = gpu.pcg(dA, b, M=gpu.Preconditioner.amg(H), control=ctl)
    x2, i2 = gpu.pcg(dA, b, M=gpu.Preconditioner.amg(G), control=ctl)
    assert (i1.iterations, i1.status) == (i2.iterations, i2.status)
    assert np.array_equal(x1.cpu().numpy(), x2.cpu().numpy(), equal_nan=True)


def test_damaged_and_foreign_files_are_refused(gpu, tmp_path):
    A = P.poisson2d(20)
    H = gpu.Hierarchy(gpu.CsrMatrix.from_arrays(*A))
    good = tmp_path / "h.bin"
    H.save(good)
    data = bytearray(good.read_bytes())
    cases = {
        "flipped": bytes(data[:100]) + bytes([data[100] ^ 0x40]) + bytes(data[101:]),
        "truncated": bytes(data[:len(data) // 2]),
        "foreign": b"not a hierarchy file at all" * 4,
    }
    for name, blob in cases.items():
        p = tmp_path / name
        p.write_bytes(blob)
        with pytest.raises(L.LabError) as e:
            gpu.Hierarchy.load(p)
        assert e.value.status == L.LAB_BAD_ARG, name
    with pytest.raises(L.LabError):
        gpu.Hierarchy.load(tmp_path / "missing.bin")
