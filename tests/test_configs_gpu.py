"""Parity at the sizes of the five benchmark workloads.

The other GPU test files check every piece on small operators; this file runs
the workloads themselves (or, where a CPU checker would take minutes, the largest
size that finishes in seconds, named in the test) and compares them with the
compiled reference (oracle/_ref, the reference's own host code) or with the C
restatement of it (oracle/oracle.c):

* 3D 7-point Poisson 128^3 (2,097,152 rows): every level A_l, P_l, R_l of the SA
  hierarchy bit-identical to the reference's saamg_setup (saamg.cpp:210-282), and
  the PCG solution against the reference's cg_solver with its V-cycle
  (cg.cpp:136-223) to 1e-7 relative, iterations within +-1.
* 3D 27-point variable-coefficient diffusion, mixed precision: the FP32 and
  FP32 + BF16 hierarchies inside the FP64 PCG against an FP64 oracle solve, at
  96^3 (884,736 rows, 23.3M entries; the oracle needs about a minute at 160^3).
* 256 uneven 2D Poisson systems (sides U{32..256}, 6.9M rows) in one batched
  solve: per-system iterations against the segmented algorithm on the CPU and
  every solution against the system solved alone by the oracle.
* 96^3 graph Laplacian adjoint: dL/db and dL/dA against the FP64 CPU gradient
  built from oracle solves, and central finite differences on 64 random
  nonzeros (symmetric pairs) and 8 entries of b.
"""
import concurrent.futures as cf

import numpy as np
import pytest
import torch

from linalglib_b200 import _lib as L
from linalglib_b200 import problems as P

from helpers import csr_diff, csr_equal, inf_rel_residual

pytestmark = [pytest.mark.gpu, pytest.mark.slow]


# ---------------------------------------------------------------- 128^3 Poisson
@pytest.fixture(scope="module")
def poisson128(gpu, reference):
    A = P.poisson3d(128)
    b, xt = P.rhs_from_solution(*A[:3], seed=0)
    dA = gpu.CsrMatrix.from_arrays(*A[:3])
    H = gpu.Hierarchy(dA, kind=L.AMG_SA)
    Hr = reference.amg_setup(A, kind=0)
    return A, b, xt, dA, H, Hr


def test_poisson128_hierarchy_bit_identical_to_reference(poisson128):
    A, b, xt, dA, H, Hr = poisson128
    assert H.levels == Hr.levels, (H.levels, Hr.levels)
    for l in range(H.levels + 1):
        g, r = H.A(l).to_numpy(), Hr.A(l)
        assert csr_equal(g, r), f"A_{l}: {csr_diff(g, r)}"
        if l < H.levels:
            for name, gm, rm in (("P", H.P(l), Hr.P(l)), ("R", H.R(l), Hr.R(l))):
                gm = gm.to_numpy()
                assert csr_equal(gm, rm), f"{name}_{l}: {csr_diff(gm, rm)}"


def test_poisson128_pcg_matches_reference_solution(gpu, poisson128):
    A, b, xt, dA, H, Hr = poisson128
    M = gpu.Preconditioner.amg(H)
    x, info = gpu.pcg(dA, gpu.vec(b), M=M,
                      control=gpu.iter_control(rel_tol=1e-8, abs_tol=0.0, max_iter=1000))
    xr, itr = Hr.pcg(b, rel_tol=1e-8, abs_tol=1e-300)
    assert info.converged == 1 and info.status == L.LAB_OK
    assert abs(info.iterations - itr) <= 1, (info.iterations, itr)
    x = x.cpu().numpy()
    assert inf_rel_residual(A, x, b) <= 1e-8 * 1.0001
    assert np.max(np.abs(x - xr)) <= 1e-7 * np.max(np.abs(xr))


# ---------------------------------------------------------------- 27-point, mixed
def test_diffusion27_96_mixed_vs_fp64_oracle(gpu, oracle):
    A = P.diffusion27(96, seed=0)
    b, _ = P.rhs_from_solution(*A[:3], seed=0)
    dA = gpu.CsrMatrix.from_arrays(*A[:3])
    H = gpu.Hierarchy(dA)
    ctl = gpu.iter_control(rel_tol=1e-10, abs_tol=0.0, max_iter=1000)
    xo, ito, _ = oracle.amg_setup(A).pcg(b, omega=2.0 / 3.0, coarse=1, rel_tol=1e-10,
                                         abs_tol=0.0, max_iter=1000)
    scale = np.max(np.abs(xo))
    x64, i64 = gpu.pcg(dA, gpu.vec(b), M=gpu.Preconditioner.amg(H, gpu.amg_options(omega=2.0 / 3.0)),
                       control=ctl)
    assert i64.converged and abs(i64.iterations - ito) <= 1, (i64.iterations, ito)
    x64 = x64.cpu().numpy()
    assert np.max(np.abs(x64 - xo)) <= 1e-8 * scale
    for prec, slack in ((L.PREC_FP32, 3), (L.PREC_FP32_BF16, max(6, ito // 2))):
        M = gpu.Preconditioner.amg(H, gpu.amg_options(omega=2.0 / 3.0, precision=prec))
        xlp, ilp = gpu.pcg(dA, gpu.vec(b), M=M, control=ctl)
        assert ilp.converged and ilp.iterations <= ito + slack, (prec, ilp.iterations, ito)
        xlp = xlp.cpu().numpy()
        # the outer FP64 CG reaches the FP64 residual; the error against the FP64
        # oracle solution is that of any 1e-10 solve of this operator
        assert inf_rel_residual(A, xlp, b) <= 1e-10 * 1.0001
        assert np.max(np.abs(xlp - xo)) <= 1e-8 * scale, (prec, np.max(np.abs(xlp - xo)) / scale)


# ---------------------------------------------------------------- 256 systems
def test_batched_256_uneven_systems(gpu, oracle):
    from test_batch_gpu import segmented_pcg_oracle
    rng = np.random.default_rng(0)
    sides = rng.integers(32, 257, size=256)
    mats = [P.poisson2d(int(s)) for s in sides]
    rhs = [P.rhs_from_solution(*A, seed=k)[0] for k, A in enumerate(mats)]
    S, offs = gpu.block_diag([gpu.CsrMatrix.from_arrays(*A) for A in mats])
    assert offs[-1] == sum(int(s) ** 2 for s in sides)
    M = gpu.Preconditioner.amg(gpu.Hierarchy(S))
    bb = np.concatenate(rhs)
    x, iters, conv, info = gpu.batched_pcg(S, offs, gpu.vec(bb), M,
                                           control=gpu.iter_control(rel_tol=1e-8, abs_tol=0.0))
    assert info.converged and conv.all()
    x = x.cpu().numpy()
    # the same segmented algorithm on the CPU over the oracle's stacked hierarchy
    Sh = S.to_numpy()
    xo, ito = segmented_pcg_oracle(oracle, oracle.amg_setup(Sh), Sh, offs, bb, 1e-8)
    assert np.all(np.abs(iters - ito) <= 1), np.nonzero(np.abs(iters - ito) > 1)

    # every system solved alone by the oracle (its own hierarchy), 16 at a time
    # (the C oracle keeps no global state and ctypes releases the GIL)
    def alone(k):
        xa, ita, _ = oracle.amg_setup(mats[k]).pcg(rhs[k], rel_tol=1e-8, abs_tol=0.0, coarse=1)
        return xa

    with cf.ThreadPoolExecutor(16) as ex:
        xs = list(ex.map(alone, range(len(mats))))
    for k, A in enumerate(mats):
        xk = x[offs[k]:offs[k + 1]]
        assert inf_rel_residual(A, xk, rhs[k]) <= 1e-8 * 1.0001, k
        assert np.max(np.abs(xk - xo[offs[k]:offs[k + 1]])) <= 1e-6 * np.max(np.abs(xk)), k
        assert np.max(np.abs(xk - xs[k])) <= 1e-6 * np.max(np.abs(xs[k])), k


# ---------------------------------------------------------------- 96^3 adjoint
def test_adjoint_96_gradient_and_finite_differences(gpu, oracle):
    n, rtol = 96, 1e-11
    rp, ci, v = P.graph_laplacian3d(n, sigma=1.0, shift=1e-3, seed=0)
    m = rp.size - 1
    b, _ = P.rhs_from_solution(rp, ci, v, seed=0)
    xt = np.random.default_rng(1).standard_normal(m)
    dev = gpu.vec
    ctl = gpu.iter_control(rel_tol=rtol, abs_tol=0.0, max_iter=2000)
    A = gpu.CsrMatrix.from_arrays(rp, ci, v)
    M = gpu.Preconditioner.amg(gpu.Hierarchy(A), gpu.amg_options(omega=2.0 / 3.0))
    x, info = gpu.pcg(A, dev(b), M=M, control=ctl)
    assert info.converged
    lam, info = gpu.adjoint_solve(A, x - dev(xt), M=M, symmetric=True, control=ctl)
    assert info.converged
    gA = gpu.adjoint_grad_A(A, lam, x).cpu().numpy()
    gb = lam.cpu().numpy()
    x = x.cpu().numpy()

    # (1) the FP64 CPU reference gradient from the oracle's solves
    h = oracle.amg_setup((rp, ci, v))
    xo, _, _ = h.pcg(b, omega=2.0 / 3.0, coarse=1, rel_tol=rtol, abs_tol=0.0, max_iter=2000)
    lo, _, _ = h.pcg(xo - xt, omega=2.0 / 3.0, coarse=1, rel_tol=rtol, abs_tol=0.0, max_iter=2000)
    rows = np.repeat(np.arange(m), np.diff(rp))
    gA_ref = -lo[rows] * xo[ci]
    assert np.max(np.abs(gb - lo)) <= 1e-7 * np.max(np.abs(lo))
    assert np.max(np.abs(gA - gA_ref)) <= 1e-7 * np.max(np.abs(gA_ref))

    # (2) central differences of L = 0.5 ||x - xt||^2 from forward solves alone.
    # Each perturbed solution is taken as x_pm = x + d_pm with A_pm d_pm = b_pm - A_pm x
    # (one refinement step from the unperturbed solution x), so the error of x
    # cancels and the 1e-11 solve tolerance applies to the small corrections d_pm;
    # L(+) - L(-) = (d+ - d-) . ((x+ + x-) / 2 - xt) exactly.
    key = rows.astype(np.int64) * m + ci
    tkey = ci.astype(np.int64) * m + rows
    order = np.argsort(key)
    tpos = order[np.searchsorted(key[order], tkey)]
    Ap = gpu.CsrMatrix.from_arrays(rp, ci, v)
    Am = gpu.CsrMatrix.from_arrays(rp, ci, v)
    vd, bd, xd, xtd = dev(v), dev(b), dev(x), dev(xt)

    def central(vp, vm, bp, bm):
        Ap.set_values(vp)
        Am.set_values(vm)
        dp, i1 = gpu.pcg(Ap, Ap.residual(xd, bp), M=M, control=ctl)
        dm, i2 = gpu.pcg(Am, Am.residual(xd, bm), M=M, control=ctl)
        assert i1.converged and i2.converged
        return float(torch.dot(dp - dm, xd + 0.5 * (dp + dm) - xtd))

    rng = np.random.default_rng(7)
    for j in rng.choice(v.size, size=64, replace=False):
        i, c = rows[j], ci[j]
        hh = 1e-6 * abs(v[j])
        idx = [int(j)] if c == i else [int(j), int(tpos[j])]  # a_ij and a_ji together
        vp, vm = vd.clone(), vd.clone()
        vp[idx] += hh
        vm[idx] -= hh
        g = sum(gA[q] for q in idx)
        fd = central(vp, vm, bd, bd) / (2 * hh)
        assert abs(fd - g) <= 1e-5 * max(1.0, abs(g)), (j, fd, g)
    for k in rng.choice(m, size=8, replace=False):
        hh = 1e-6 * max(1.0, abs(b[k]))
        bp, bm = bd.clone(), bd.clone()
        bp[int(k)] += hh
        bm[int(k)] -= hh
        fd = central(vd, vd, bp, bm) / (2 * hh)
        assert abs(fd - gb[k]) <= 1e-5 * max(1.0, abs(gb[k])), (k, fd, gb[k])
