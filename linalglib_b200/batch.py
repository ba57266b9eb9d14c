"""Independent systems split over the GPUs of a job (one process per GPU).

The systems of a batch do not couple, so the multi-GPU form needs no collective
on the data path: every rank takes its share by a size-balanced partition
(lab_batch_partition: largest system first, to the least-loaded rank), solves it
on its own GPU as one batched solve, and the per-system results are gathered to
rank 0 on the host at the end.

``solve_share(mats, rhs)`` is the per-rank solver: it receives the rank's systems
and returns, for each, (x, iterations, converged).  ``solve_on_device`` is the
GPU one (block-diagonal stack, one SA hierarchy, the segmented batched PCG).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib as L


def partition(costs, nparts):
    """part[k] for each system, by lab_batch_partition."""
    costs = np.ascontiguousarray(costs, dtype=np.int64)
    part = np.zeros(costs.size, dtype=np.int32)
    L.call("lab_batch_partition", int(costs.size), C.c_void_p(costs.ctypes.data), int(nparts),
           C.c_void_p(part.ctypes.data))
    return part


def solve_on_device(mats, rhs, rel_tol=1e-8, omega=2.0 / 3.0):
    """One batched solve of this rank's systems on its GPU."""
    import linalglib_b200.core as core
    if not mats:
        return []
    blocks = [core.CsrMatrix.from_arrays(*A[:3]) for A in mats]
    S, offs = core.block_diag(blocks)
    M = core.Preconditioner.amg(core.Hierarchy(S), core.amg_options(omega=omega))
    x, iters, conv, _ = core.batched_pcg(S, offs, core.vec(np.concatenate(rhs)), M,
                                         control=core.iter_control(rel_tol=rel_tol, abs_tol=0.0))
    x = x.cpu().numpy()
    return [(x[offs[k]:offs[k + 1]].copy(), int(iters[k]), bool(conv[k]))
            for k in range(len(mats))]


def solve_partitioned(mats, rhs, solve_share, rank=0, world=1, dist=None):
    """Solve every system: this rank's share locally, then gather all results to
    rank 0 (torch.distributed object gather; the process group may be gloo or
    nccl).  Returns the list of (x, iterations, converged) in system order on
    rank 0 and None elsewhere; with world == 1 no process group is used."""
    costs = [int(A[0][-1]) + A[0].size - 1 for A in mats]  # nonzeros + rows
    part = partition(costs, world)
    mine = [k for k in range(len(mats)) if part[k] == rank]
    local = solve_share([mats[k] for k in mine], [rhs[k] for k in mine])
    pieces = list(zip(mine, local))
    if world == 1:
        gathered = [pieces]
    else:
        gathered = [None] * world if rank == 0 else None
        dist.gather_object(pieces, gathered, dst=0)
    if rank != 0:
        return None
    out = [None] * len(mats)
    for share in gathered:
        for k, res in share:
            out[k] = res
    assert all(r is not None for r in out)
    return out
