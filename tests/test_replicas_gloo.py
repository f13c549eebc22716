"""bench.py's multi-rank plumbing on CPU: two gloo ranks (127.0.0.1), the
max-over-ranks timing collective, the whole-job value of weak-scaling
replicas, and the reference arm printing on rank 0 only."""
import os
import socket
import subprocess
import sys

import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

WORKER = r"""
import datetime, os, sys
sys.path.insert(0, {repo!r})
import torch.distributed as dist
import bench
rank, local, world = bench.dist_env()
dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=60))
ms = [2.5, 4.0][rank]
m = bench.max_over_ranks(ms, world, "cpu")
v = bench.replicas_value(m, 32, world)
dist.barrier()
print(f"RANK{{rank}} {{m}} {{v}}", flush=True)
dist.destroy_process_group()
"""


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def test_two_gloo_ranks_take_the_max_and_sum_replicas(tmp_path):
    script = tmp_path / "worker.py"
    script.write_text(WORKER.format(repo=REPO))
    port = _free_port()
    procs = []
    for rank in range(2):
        env = dict(os.environ, RANK=str(rank), LOCAL_RANK=str(rank), WORLD_SIZE="2", MASTER_ADDR="127.0.0.1",
                   MASTER_PORT=str(port))
        procs.append(subprocess.Popen([sys.executable, str(script)], env=env, stdout=subprocess.PIPE,
                                      stderr=subprocess.STDOUT, text=True))
    outs = []
    for p in procs:
        out, _ = p.communicate(timeout=120)
        assert p.returncode == 0, out
        outs.append(out)
    for rank, out in enumerate(outs):
        line = [l for l in out.splitlines() if l.startswith(f"RANK{rank}")][0]
        _, m, v = line.split()
        assert float(m) == 4.0                      # the slower rank's time
        assert float(v) == 2 * 32 * 1000.0 / 4.0    # two replicas, whole-job q/s


def test_reference_arm_prints_on_rank_zero_only():
    env = dict(os.environ, RANK="1", LOCAL_RANK="1", WORLD_SIZE="2")
    p = subprocess.run([sys.executable, os.path.join(REPO, "bench.py"), "--impl", "reference", "--steps", "1",
                        "--warmup", "1"], env=env, capture_output=True, text=True, timeout=120)
    assert p.returncode == 0, p.stderr
    assert p.stdout.strip() == ""
