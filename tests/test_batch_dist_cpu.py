"""The batched workload split over GPUs, on the CPU: the size-balanced partition
(lab_batch_partition, host only) and the world-size-2 gather of per-rank solves
over gloo.  Each rank solves its share with the C oracle (the GPU ranks run the
library's batched PCG instead); rank 0 must end up with every system's solution,
identical to solving them all in one process."""
import json
import os
import socket
import subprocess
import sys

import numpy as np

from linalglib_b200 import batch
from linalglib_b200 import problems as P

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_partition_is_balanced_and_deterministic():
    rng = np.random.default_rng(0)
    sides = rng.integers(32, 257, size=256)
    costs = sides.astype(np.int64) ** 2
    for nparts in (1, 2, 3, 4, 8):
        part = batch.partition(costs, nparts)
        assert part.min() >= 0 and part.max() < nparts
        assert np.array_equal(part, batch.partition(costs, nparts))
        loads = np.bincount(part, weights=costs, minlength=nparts)
        # the greedy rule keeps every worker within the largest system of the mean
        assert loads.max() - loads.min() <= costs.max()
        assert loads.max() <= costs.sum() / nparts + costs.max()


def test_partition_edge_cases():
    assert batch.partition([], 4).size == 0
    assert list(batch.partition([5], 3)) == [0]
    # equal costs alternate over the workers in input order
    assert list(batch.partition([7, 7, 7, 7], 2)) == [0, 1, 0, 1]
    assert list(batch.partition([1, 9, 4], 2)) == [1, 0, 1]


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


_WORKER = r"""
import os, sys, json
sys.path.insert(0, os.environ["LAB_ROOT"])
import numpy as np
import torch.distributed as dist
from linalglib_b200 import batch, problems as P
from oracle.oracle import Oracle

rank, world = int(os.environ["RANK"]), int(os.environ["WORLD_SIZE"])
if world > 1:
    dist.init_process_group("gloo")
rng = np.random.default_rng(3)
sides = rng.integers(6, 20, size=9)
mats = [P.poisson2d(int(s)) for s in sides]
rhs = [P.rhs_from_solution(*A, seed=k)[0] for k, A in enumerate(mats)]
O = Oracle()

def oracle_share(ms, bs):
    out = []
    for A, b in zip(ms, bs):
        x, it, _ = O.amg_setup(A).pcg(b, rel_tol=1e-8, abs_tol=0.0, coarse=1)
        out.append((x, it, True))
    return out

res = batch.solve_partitioned(mats, rhs, oracle_share, rank=rank, world=world,
                              dist=dist if world > 1 else None)
if rank == 0:
    np.save(os.environ["LAB_OUT"], np.concatenate([r[0] for r in res]))
    print(json.dumps({"iters": [r[1] for r in res]}), flush=True)
if world > 1:
    dist.destroy_process_group()
"""


def _run(tmp_path, world):
    script = tmp_path / "worker.py"
    script.write_text(_WORKER)
    port = _free_port()
    out = tmp_path / f"x{world}.npy"
    procs = []
    for rank in range(world):
        env = dict(os.environ, RANK=str(rank), LOCAL_RANK=str(rank), WORLD_SIZE=str(world),
                   MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), LAB_ROOT=ROOT, LAB_OUT=str(out))
        procs.append(subprocess.Popen([sys.executable, str(script)], env=env,
                                      stdout=subprocess.PIPE, stderr=subprocess.PIPE, text=True))
    outs = [p.communicate(timeout=300) for p in procs]
    for p, (o, e) in zip(procs, outs):
        assert p.returncode == 0, e[-3000:]
    line = json.loads(outs[0][0].strip().splitlines()[-1])
    return np.load(out), line["iters"]


def test_partitioned_solve_gathers_every_system_gloo(tmp_path):
    x2, it2 = _run(tmp_path, 2)
    x1, it1 = _run(tmp_path, 1)
    assert it2 == it1
    assert np.array_equal(x2, x1)
