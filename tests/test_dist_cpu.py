"""The multi-process paths of bench.py on the CPU (gloo, world size 2): the
rank bookkeeping and the max-over-ranks timing reduction, and the reference arm
under torchrun (rank 0 alone runs the reference and prints the line; the other
rank exits 0 without work)."""
import json
import os
import socket
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


_WORKER = r"""
import os, sys, json
sys.path.insert(0, os.environ["LAB_ROOT"])
import bench
d = bench.Dist()
d.init(need_gpu=False)
d.barrier()
v = d.max(1.5 + d.rank)
print(json.dumps({"rank": d.rank, "world": d.world, "max": v}), flush=True)
d.close()
"""


def test_dist_max_over_ranks_gloo(tmp_path):
    script = tmp_path / "worker.py"
    script.write_text(_WORKER)
    port = _free_port()
    procs = []
    for rank in range(2):
        env = dict(os.environ, RANK=str(rank), LOCAL_RANK=str(rank), WORLD_SIZE="2",
                   MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), LAB_ROOT=ROOT)
        procs.append(subprocess.Popen([sys.executable, str(script)], env=env,
                                      stdout=subprocess.PIPE, stderr=subprocess.PIPE, text=True))
    outs = [p.communicate(timeout=120) for p in procs]
    for p, (o, e) in zip(procs, outs):
        assert p.returncode == 0, e
    lines = [json.loads(o.strip().splitlines()[-1]) for o, _ in outs]
    assert sorted(l["rank"] for l in lines) == [0, 1]
    assert all(l["world"] == 2 and l["max"] == 2.5 for l in lines)


def test_reference_arm_two_ranks_torchrun():
    # (--grid: torchrun's own parser would take --n as an abbreviation)
    if not os.path.exists(os.path.join(ROOT, "oracle", "_ref", "liblinalg_ref.so")):
        pytest.skip("compiled reference not built")
    port = _free_port()
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", str(port), "bench.py", "--impl",
           "reference", "--gpus", "2", "--grid", "12", "--steps", "1", "--warmup", "1"]
    r = subprocess.run(cmd, cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [l for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1, r.stdout
    line = json.loads(lines[0])
    assert line["impl"] == "reference" and line["value"] > 0
    assert line["e2e"]["h2d_bytes_per_step"] == 0 and line["cpu_baseline"]["kind"] == "reference"
