"""Batched solves: many uneven independent systems in one stacked solve with a
per-system convergence mask, and block PCG over many right-hand sides.  Each
system / column must behave as if it had been solved alone: same stopping test,
iteration counts within +-1 of the single-system oracle solve, solutions within
the tolerance.
"""
import numpy as np
import pytest
import torch

from linalglib_b200 import _lib as L
from linalglib_b200 import problems as P

from helpers import inf_rel_residual

pytestmark = pytest.mark.gpu


def test_block_diag_and_hierarchy_decouple(gpu, oracle):
    sides = [9, 14, 11]
    mats = [P.poisson2d(s) for s in sides]
    blocks = [gpu.CsrMatrix.from_arrays(*A) for A in mats]
    S, offs = gpu.block_diag(blocks)
    assert list(offs) == list(np.cumsum([0] + [s * s for s in sides]))
    rp, ci, v, _ = S.to_numpy()
    for k, A in enumerate(mats):
        r0, r1 = offs[k], offs[k + 1]
        sub_rp = rp[r0:r1 + 1] - rp[r0]
        assert np.array_equal(sub_rp, A[0])
        assert np.array_equal(ci[rp[r0]:rp[r1]] - r0, A[1])
    # the stacked hierarchy never couples blocks: every level is block diagonal
    H = gpu.Hierarchy(S)
    for l in range(H.levels):
        p = H.P(l).to_numpy()
        assert p[0][-1] == p[1].size


def segmented_pcg_oracle(oracle, Hs, S, offs, b, rtol, max_iter=1000):
    """The batched algorithm on the CPU: per-segment CG scalars (cg.cpp:136-223 for
    every system) with the oracle's V-cycle on the stacked hierarchy."""
    nseg = len(offs) - 1
    seg = [slice(offs[k], offs[k + 1]) for k in range(nseg)]
    x = np.zeros_like(b)
    r = b.copy()
    r0 = np.array([np.max(np.abs(r[s])) for s in seg])
    z = Hs.vcycle(r, coarse=1)
    p = z.copy()
    gamma = np.array([np.dot(z[s], r[s]) for s in seg])
    done = r0 == 0
    iters = np.zeros(nseg, dtype=int)
    for _ in range(max_iter + 1):
        if done.all():
            break
        q = oracle.spmv(S, p)
        for k, s in enumerate(seg):
            if done[k]:
                continue
            alpha = gamma[k] / np.dot(q[s], p[s])
            x[s] = alpha * p[s] + x[s]
            r[s] = (-1.0 * alpha) * q[s] + r[s]
            if np.max(np.abs(r[s])) / r0[k] <= rtol:
                done[k] = True
        if done.all():
            break
        z = Hs.vcycle(r, coarse=1)
        for k, s in enumerate(seg):
            if done[k]:
                continue
            g = np.dot(z[s], r[s])
            p[s] = z[s] + (g / gamma[k]) * p[s]
            gamma[k] = g
            iters[k] += 1
    return x, iters


@pytest.mark.parametrize("nsys", [5, 40])
def test_batched_pcg_matches_oracle(gpu, oracle, nsys):
    rng = np.random.default_rng(nsys)
    sides = rng.integers(8, 48, size=nsys)
    mats = [P.poisson2d(int(s)) for s in sides]
    rhs = [P.rhs_from_solution(*A, seed=k)[0] for k, A in enumerate(mats)]
    blocks = [gpu.CsrMatrix.from_arrays(*A) for A in mats]
    S, offs = gpu.block_diag(blocks)
    H = gpu.Hierarchy(S)
    M = gpu.Preconditioner.amg(H)
    bb = np.concatenate(rhs)
    x, iters, conv, info = gpu.batched_pcg(S, offs, gpu.vec(bb), M,
                                           control=gpu.iter_control(rel_tol=1e-8, abs_tol=0.0))
    assert info.converged and conv.all()
    x = x.cpu().numpy()
    Sh = S.to_numpy()
    xo, ito = segmented_pcg_oracle(oracle, oracle.amg_setup(Sh), Sh, offs, bb, 1e-8)
    assert np.all(np.abs(iters - ito) <= 1), (iters, ito)
    for k, A in enumerate(mats):
        xk = x[offs[k]:offs[k + 1]]
        assert inf_rel_residual(A, xk, rhs[k]) <= 1e-8 * 1.0001
        xs = xo[offs[k]:offs[k + 1]]
        assert np.max(np.abs(xk - xs)) <= 1e-6 * np.max(np.abs(xs))
        # and the same answer as solving the system alone
        xa, _, _ = oracle.amg_setup(A).pcg(rhs[k], rel_tol=1e-8, abs_tol=0.0, coarse=1)
        assert np.max(np.abs(xk - xa)) <= 1e-6 * np.max(np.abs(xa))


def test_batched_mask_keeps_converged_systems_fixed(gpu):
    """A system converging early must not move while the others iterate."""
    A1, A2 = P.poisson2d(8), P.poisson2d(40)
    b1 = np.zeros(64)  # converged at iteration 0
    b2, _ = P.rhs_from_solution(*A2, seed=1)
    S, offs = gpu.block_diag([gpu.CsrMatrix.from_arrays(*A1), gpu.CsrMatrix.from_arrays(*A2)])
    M = gpu.Preconditioner.amg(gpu.Hierarchy(S))
    x, iters, conv, info = gpu.batched_pcg(S, offs, gpu.vec(np.concatenate([b1, b2])), M,
                                           control=gpu.iter_control(rel_tol=1e-9, abs_tol=0.0))
    assert conv.all() and iters[0] == 0 and iters[1] > 5
    assert torch.count_nonzero(x[:64]) == 0


def test_multi_rhs_pcg(gpu, oracle):
    A = P.poisson3d(16)
    n = A[0].size - 1
    k = 11
    B = np.random.default_rng(4).uniform(-1, 1, (k, n))
    dA = gpu.CsrMatrix.from_arrays(*A)
    M = gpu.Preconditioner.amg(gpu.Hierarchy(dA))
    X, iters, conv, info = gpu.multi_rhs_pcg(dA, gpu.vec(B).reshape(k, n), M,
                                             control=gpu.iter_control(rel_tol=1e-8, abs_tol=0.0))
    assert info.converged and conv.all()
    X = X.cpu().numpy()
    h = oracle.amg_setup(A)
    for j in range(k):
        assert inf_rel_residual(A, X[j], B[j]) <= 1e-8 * 1.0001
        xo, ito, _ = h.pcg(B[j], rel_tol=1e-8, abs_tol=0.0, coarse=1)
        assert abs(int(iters[j]) - ito) <= 1
        assert np.max(np.abs(X[j] - xo)) <= 1e-6 * np.max(np.abs(xo))
