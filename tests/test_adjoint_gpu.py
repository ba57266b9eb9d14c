"""Adjoint path: dL/db and dL/dA (on the sparsity pattern) of x = A^{-1} b for
L = 0.5 ||x - x_target||^2 on the weighted 3D graph Laplacian (+1e-3 shift),
through the C ABI, wrapped in a torch.autograd.Function here in the tests only.

Checked against (1) an FP64 CPU reference gradient built from the oracle's own
solves (forward PCG, adjoint PCG, -lambda_i x_j) and (2) central finite
differences on 64 random nonzeros (symmetric pairs a_ij, a_ji perturbed
together, since CG needs a symmetric operator) and on entries of b.  The forward
iterates are never stored: backward() rebuilds the hierarchy and solves again.
"""
import numpy as np
import pytest
import torch

from linalglib_b200 import problems as P

pytestmark = pytest.mark.gpu

RTOL = 1e-12


def _solve(core, rp, ci, vals, b):
    A = core.CsrMatrix.from_arrays(rp, ci, vals)
    H = core.Hierarchy(A)
    M = core.Preconditioner.amg(H, core.amg_options(omega=2.0 / 3.0))
    x, info = core.pcg(A, b, M=M, control=core.iter_control(rel_tol=RTOL, abs_tol=0.0,
                                                              max_iter=2000))
    assert info.converged
    return A, M, x


class AmgSolve(torch.autograd.Function):
    """x = A(vals)^{-1} b with the pattern (rp, ci) fixed."""

    @staticmethod
    def forward(ctx, vals, b, rp, ci, core):
        A, M, x = _solve(core, rp, ci, vals.detach().contiguous(), b.detach().contiguous())
        ctx.save_for_backward(vals, x)
        ctx.rp, ctx.ci, ctx.core = rp, ci, core
        return x

    @staticmethod
    def backward(ctx, gx):
        vals, x = ctx.saved_tensors
        core = ctx.core
        # recompute the operator and its preconditioner (nothing of the forward solve kept)
        A = core.CsrMatrix.from_arrays(ctx.rp, ctx.ci, vals.detach().contiguous())
        H = core.Hierarchy(A)
        M = core.Preconditioner.amg(H, core.amg_options(omega=2.0 / 3.0))
        lam, info = core.adjoint_solve(A, gx.contiguous(), M=M, symmetric=True,
                                       control=core.iter_control(rel_tol=RTOL, abs_tol=0.0,
                                                                 max_iter=2000))
        assert info.converged
        gA = core.adjoint_grad_A(A, lam, x)
        return gA, lam, None, None, None


def _loss(x, xt):
    return 0.5 * torch.sum((x - xt) ** 2)


@pytest.fixture(scope="module")
def system():
    n = 12
    rp, ci, v = P.graph_laplacian3d(n, sigma=1.0, shift=1e-3, seed=0)
    b, _ = P.rhs_from_solution(rp, ci, v, seed=0)
    xt = np.random.default_rng(1).standard_normal(rp.size - 1)
    return rp, ci, v, b, xt


def test_adjoint_matches_cpu_reference_gradient(gpu, oracle, system):
    rp, ci, v, b, xt = system
    core = gpu
    vals = torch.tensor(v, device="cuda", requires_grad=True)
    bt = torch.tensor(b, device="cuda", requires_grad=True)
    x = AmgSolve.apply(vals, bt, torch.as_tensor(rp, device="cuda"),
                       torch.as_tensor(ci, device="cuda"), core)
    L = _loss(x, torch.as_tensor(xt, device="cuda"))
    L.backward()
    # FP64 CPU reference: x = A^-1 b, lambda = A^-1 (x - xt), dL/dA_ij = -lambda_i x_j
    h = oracle.amg_setup((rp, ci, v))
    xo, _, _ = h.pcg(b, omega=2.0 / 3.0, coarse=1, rel_tol=RTOL, abs_tol=0.0, max_iter=2000)
    lo, _, _ = h.pcg(xo - xt, omega=2.0 / 3.0, coarse=1, rel_tol=RTOL, abs_tol=0.0, max_iter=2000)
    rows = np.repeat(np.arange(rp.size - 1), np.diff(rp))
    gA_ref = -lo[rows] * xo[ci]
    gb = bt.grad.cpu().numpy()
    gA = vals.grad.cpu().numpy()
    assert np.max(np.abs(gb - lo)) <= 1e-8 * np.max(np.abs(lo))
    assert np.max(np.abs(gA - gA_ref)) <= 1e-8 * np.max(np.abs(gA_ref))


def test_adjoint_finite_differences(gpu, system):
    rp, ci, v, b, xt = system
    core = gpu
    m = rp.size - 1
    dev = lambda a: torch.as_tensor(a, device="cuda")
    vals = torch.tensor(v, device="cuda", requires_grad=True)
    bt = torch.tensor(b, device="cuda", requires_grad=True)
    x = AmgSolve.apply(vals, bt, dev(rp), dev(ci), core)
    _loss(x, dev(xt)).backward()
    gA = vals.grad.cpu().numpy()
    gb = bt.grad.cpu().numpy()

    def L_of(vv, bb):
        _, _, xx = _solve(core, rp, ci, dev(vv), dev(bb))
        return float(_loss(xx, dev(xt)))

    rows = np.repeat(np.arange(m), np.diff(rp))
    # index of the transposed entry (j, i) for every stored (i, j)
    key = rows.astype(np.int64) * m + ci
    tkey = ci.astype(np.int64) * m + rows
    order = np.argsort(key)
    tpos = order[np.searchsorted(key[order], tkey)]
    rng = np.random.default_rng(7)
    picks = rng.choice(v.size, size=64, replace=False)
    for j in picks:
        i, c = rows[j], ci[j]
        h = 1e-5 * abs(v[j])
        vp, vm = v.copy(), v.copy()
        if c == i:
            vp[j] += h
            vm[j] -= h
            g = gA[j]
        else:
            vp[j] += h
            vp[tpos[j]] += h
            vm[j] -= h
            vm[tpos[j]] -= h
            g = gA[j] + gA[tpos[j]]
        fd = (L_of(vp, b) - L_of(vm, b)) / (2 * h)
        assert abs(fd - g) <= 1e-4 * max(1.0, abs(g)), (j, fd, g)
    for k in rng.choice(m, size=8, replace=False):
        h = 1e-5 * max(1.0, abs(b[k]))
        bp, bm = b.copy(), b.copy()
        bp[k] += h
        bm[k] -= h
        fd = (L_of(v, bp) - L_of(v, bm)) / (2 * h)
        assert abs(fd - gb[k]) <= 1e-4 * max(1.0, abs(gb[k])), (k, fd, gb[k])


def test_adjoint_nonsymmetric_uses_transpose(gpu, oracle):
    """Non-symmetric A: lambda solves A^T lambda = g (GMRES on the transpose)."""
    rp, ci, v = P.poisson2d(20)
    v = v.copy()
    rows = np.repeat(np.arange(rp.size - 1), np.diff(rp))
    v[ci == rows + 1] *= 0.5  # break symmetry, keep diagonal dominance
    A = gpu.CsrMatrix.from_arrays(rp, ci, v)
    g = np.random.default_rng(3).uniform(-1, 1, rp.size - 1)
    lam, info = gpu.adjoint_solve(A, gpu.vec(g), M=None, symmetric=False,
                                  control=gpu.iter_control(rel_tol=1e-11, abs_tol=0.0, max_iter=500))
    assert info.converged
    T = oracle.transpose((rp, ci, v, rp.size - 1))
    r = g - oracle.spmv(T, lam.cpu().numpy())
    assert np.max(np.abs(r)) <= 1e-9 * np.max(np.abs(g))
