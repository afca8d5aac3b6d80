"""The bench's multi-GPU host logic on CPU: two ranks over gloo (the
replicas path of `bench.py --gpus 2`, without GPUs): the job's rays are
the ranks' sum, its device time the slowest rank's, and ranks render
disjoint sample ranges; the reference arm runs on rank 0 only."""

import json
import os
import socket
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

RANK_SCRIPT = r"""
import json, os, sys
sys.path.insert(0, sys.argv[1])
import torch.distributed as dist
import bench
rank, world = int(os.environ["RANK"]), int(os.environ["WORLD_SIZE"])
dist.init_process_group("gloo", timeout=__import__("datetime").timedelta(seconds=60))
rays, e2e_rays = 1000.0 * (rank + 1), 900.0 * (rank + 1)
ms, e2e_ms = 10.0 + 5.0 * rank, 12.0 + 1.0 * rank
out = bench.reduce_over_ranks(rays, e2e_rays, ms, e2e_ms, world, "cpu")
dist.barrier()
dist.destroy_process_group()
if rank == 0:
    with open(sys.argv[2], "w") as f:
        json.dump({"totals": out, "bases": [bench.rank_sample_base(r) for r in range(world)]}, f)
"""


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_two_ranks_reduce_over_gloo(tmp_path):
    script = tmp_path / "rank.py"
    script.write_text(RANK_SCRIPT)
    out = tmp_path / "out.json"
    port = str(free_port())
    procs = []
    for rank in range(2):
        env = dict(os.environ, RANK=str(rank), WORLD_SIZE="2", LOCAL_RANK=str(rank),
                   MASTER_ADDR="127.0.0.1", MASTER_PORT=port)
        procs.append(subprocess.Popen([sys.executable, str(script), ROOT, str(out)], env=env))
    codes = [p.wait(timeout=120) for p in procs]
    assert codes == [0, 0]
    got = json.loads(out.read_text())
    assert got["totals"] == [3000.0, 2700.0, 15.0, 13.0]
    # Sample ranges of 20 + 3 + 20 + 2 frames of 16 samples never overlap.
    b0, b1 = got["bases"]
    assert b1 - b0 > 45 * 16


def test_reference_arm_runs_on_rank_zero_only(capsys):
    sys.path.insert(0, ROOT)
    import bench

    class Args:
        gpus, steps, warmup = 2, 1, 0

    assert bench.run_reference(Args(), rank=1) is None
    assert capsys.readouterr().out == ""
