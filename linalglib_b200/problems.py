"""Seeded synthetic sparse systems with the shapes of the AMG-PCG workloads.

The reference's own test fixtures are SuiteSparse ``.mtx`` files fetched over the
network (clients/matrices/matrix_downloader.py), so the workloads here are
generated: Dirichlet finite-difference Poisson operators, a 27-point
variable-coefficient diffusion operator (lognormal link conductances, z anisotropy),
and a weighted 7-point graph Laplacian.  Every matrix is CSR with int32 indices, float64
values and column indices sorted ascending inside each row (the layout the
reference's read_mtx and SpGEMM produce, library/src/csr_matrix.cpp:524-729).

Right-hand sides are b = A @ x_true with x_true ~ U[-1, 1] drawn from
``numpy.random.default_rng(seed)``.
"""
from __future__ import annotations

import numpy as np

__all__ = [
    "poisson2d",
    "poisson3d",
    "diffusion27",
    "graph_laplacian3d",
    "rhs_from_solution",
    "csr_matvec",
    "uniform_solution",
]


def _stencil_csr(shape, offsets, weights):
    """Assemble a constant/variable stencil operator on a Dirichlet grid.

    shape   -- grid extents (nz, ny, nx) or (ny, nx); the row index of grid point
               (z, y, x) is (z*ny + y)*nx + x.
    offsets -- list of integer offset tuples, one per stencil point.
    weights -- list of arrays (or scalars) with the value for each offset, shaped
               like the grid.
    Neighbours outside the grid are dropped (Dirichlet).  Offsets are sorted by
    their linear index so that each row's columns come out ascending.
    """
    shape = tuple(int(s) for s in shape)
    nd = len(shape)
    m = int(np.prod(shape))
    strides = [int(np.prod(shape[d + 1:])) for d in range(nd)]
    lin = [sum(o[d] * strides[d] for d in range(nd)) for o in offsets]
    order = np.argsort(lin, kind="stable")
    idx = np.indices(shape).reshape(nd, -1)
    rows = np.arange(m, dtype=np.int64)
    valid = []
    vals = []
    for k in order:
        o = offsets[k]
        ok = np.ones(m, dtype=bool)
        for d in range(nd):
            if o[d] < 0:
                ok &= idx[d] >= -o[d]
            elif o[d] > 0:
                ok &= idx[d] < shape[d] - o[d]
        w = weights[k]
        w = np.broadcast_to(np.asarray(w, dtype=np.float64), shape).reshape(-1)
        valid.append(ok)
        vals.append(w)
    valid = np.stack(valid, axis=1)  # (m, npts) in ascending-column order
    vals = np.stack(vals, axis=1)
    cols = rows[:, None] + np.asarray([lin[k] for k in order], dtype=np.int64)[None, :]
    counts = valid.sum(axis=1)
    row_ptr = np.zeros(m + 1, dtype=np.int64)
    np.cumsum(counts, out=row_ptr[1:])
    col_ind = cols[valid].astype(np.int32)
    val = vals[valid].astype(np.float64)
    if row_ptr[-1] >= 2**31:
        raise ValueError("matrix has more than 2^31-1 nonzeros")
    return row_ptr.astype(np.int32), col_ind, val


def poisson2d(nx: int, ny: int | None = None):
    """5-point Laplacian on an nx-by-ny grid: diagonal 4, neighbours -1."""
    ny = nx if ny is None else ny
    offs = [(0, 0), (-1, 0), (1, 0), (0, -1), (0, 1)]
    w = [4.0, -1.0, -1.0, -1.0, -1.0]
    return _stencil_csr((ny, nx), offs, w)


def poisson3d(n: int, ny: int | None = None, nz: int | None = None):
    """7-point Laplacian on an n^3 grid: diagonal 6, neighbours -1."""
    ny = n if ny is None else ny
    nz = n if nz is None else nz
    offs = [(0, 0, 0), (-1, 0, 0), (1, 0, 0), (0, -1, 0), (0, 1, 0), (0, 0, -1), (0, 0, 1)]
    w = [6.0] + [-1.0] * 6
    return _stencil_csr((nz, ny, n), offs, w)


def diffusion27(n: int, sigma: float = 1.5, zscale: float = 100.0, seed: int = 0):
    """27-point variable-coefficient diffusion operator on an n^3 Dirichlet grid.

    Every node is linked to its 26 neighbours (faces, edges, corners).  Link
    p -> p+d carries a conductance  k * (dx^2 + dy^2 + zscale*dz^2) / |d|^4  with
    k ~ lognormal(0, sigma) drawn per link (the tensor diag(1, 1, zscale) projected
    on the link direction, over the squared link length).  Row p holds -c for each
    neighbour inside the grid and the sum of all 26 link conductances on the
    diagonal (links to the eliminated boundary nodes included), so the operator is
    a symmetric, weakly diagonally dominant M-matrix (positive definite, and
    lambda_max(D^-1 A) <= 2).

    Conductances are drawn link by link from numpy.random.default_rng(seed), one
    (n+2)^3 array per half-direction d, in the order the 13 half-directions with
    d > 0 lexicographically (dz, dy, dx) are enumerated.
    """
    rng = np.random.default_rng(seed)
    halves = [(dz, dy, dx) for dz in (-1, 0, 1) for dy in (-1, 0, 1) for dx in (-1, 0, 1)
              if (dz, dy, dx) > (0, 0, 0)]
    diag = np.zeros((n, n, n))
    offs = []
    weights = []
    for d in halves:
        dz, dy, dx = d
        scale = (dx * dx + dy * dy + zscale * dz * dz) / float(dx * dx + dy * dy + dz * dz) ** 2
        # conductance of the link from padded node q (grid node q - 1) to q + d
        c = scale * rng.lognormal(0.0, sigma, size=(n + 2, n + 2, n + 2))
        fwd = c[1:n + 1, 1:n + 1, 1:n + 1]                                 # p -> p + d
        bwd = c[1 - dz:n + 1 - dz, 1 - dy:n + 1 - dy, 1 - dx:n + 1 - dx]   # p - d -> p
        diag += fwd + bwd
        offs += [d, (-dz, -dy, -dx)]
        weights += [-fwd, -bwd]
    offs.append((0, 0, 0))
    weights.append(diag)
    return _stencil_csr((n, n, n), offs, weights)


def graph_laplacian3d(n: int, sigma: float = 1.0, shift: float = 1e-3, seed: int = 0):
    """Weighted graph Laplacian of the n^3 7-point lattice plus shift*I.

    Edge conductances are lognormal(0, sigma); row i holds -w_ij off the diagonal
    and shift + sum_j w_ij on it, so the operator is symmetric positive definite.
    """
    rng = np.random.default_rng(seed)
    wx = rng.lognormal(0.0, sigma, size=(n, n, n - 1))
    wy = rng.lognormal(0.0, sigma, size=(n, n - 1, n))
    wz = rng.lognormal(0.0, sigma, size=(n - 1, n, n))

    def pad(a, axis, lo):
        padw = [(0, 0)] * 3
        padw[axis] = (1, 0) if lo else (0, 1)
        return np.pad(a, padw)

    w_xm = pad(wx, 2, True)   # edge to x-1
    w_xp = pad(wx, 2, False)  # edge to x+1
    w_ym = pad(wy, 1, True)
    w_yp = pad(wy, 1, False)
    w_zm = pad(wz, 0, True)
    w_zp = pad(wz, 0, False)
    diag = shift + w_xm + w_xp + w_ym + w_yp + w_zm + w_zp
    offs = [(0, 0, 0), (0, 0, -1), (0, 0, 1), (0, -1, 0), (0, 1, 0), (-1, 0, 0), (1, 0, 0)]
    weights = [diag, -w_xm, -w_xp, -w_ym, -w_yp, -w_zm, -w_zp]
    return _stencil_csr((n, n, n), offs, weights)


def csr_matvec(row_ptr, col_ind, val, x):
    """y = A @ x on the host with numpy (used only to build right-hand sides)."""
    row_ptr = np.asarray(row_ptr)
    m = row_ptr.size - 1
    prod = np.asarray(val) * np.asarray(x)[np.asarray(col_ind)]
    rows = np.repeat(np.arange(m), np.diff(row_ptr))
    return np.bincount(rows, weights=prod, minlength=m).astype(np.float64)


def uniform_solution(m: int, seed: int = 0):
    """x_true ~ U[-1, 1] from numpy.random.default_rng(seed)."""
    return np.random.default_rng(seed).uniform(-1.0, 1.0, size=m)


def rhs_from_solution(row_ptr, col_ind, val, seed: int = 0):
    """(b, x_true) with b = A @ x_true, x_true ~ U[-1, 1]."""
    x = uniform_solution(len(row_ptr) - 1, seed)
    return csr_matvec(row_ptr, col_ind, val, x), x
