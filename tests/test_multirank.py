"""The multi-rank logic of bench.py (replicas, weak scaling) on CPU with
gloo, world size 2: every rank gets the slowest rank's time, the whole-job
rate counts every rank's units, and only rank 0 runs the reference arm."""
import os
import socket
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

WORKER = r"""
import os, sys, io, contextlib
sys.path.insert(0, {root!r})
import torch.distributed as dist
from datetime import timedelta
import bench
rank = int(os.environ["RANK"]); world = int(os.environ["WORLD_SIZE"])
dist.init_process_group("gloo", timeout=timedelta(seconds=60))
ms = bench.max_over_ranks(10.0 + 5.0 * rank, world, "cpu")
assert ms == 15.0, ms
assert bench.aggregate_rate(1000, world, ms) == 2 * 1000 / 0.015
class A: steps = 1; warmup = 0; gpus = world
buf = io.StringIO()
if rank == 1:
    with contextlib.redirect_stdout(buf):
        bench.run_reference(A, rank, world)
    assert buf.getvalue() == "", buf.getvalue()
dist.barrier()
dist.destroy_process_group()
print("rank", rank, "ok")
"""


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def test_two_gloo_ranks(tmp_path):
    pytest.importorskip("torch")
    script = tmp_path / "worker.py"
    script.write_text(WORKER.format(root=ROOT))
    port = _free_port()
    procs = []
    for rank in range(2):
        env = dict(os.environ, RANK=str(rank), WORLD_SIZE="2", LOCAL_RANK=str(rank), MASTER_ADDR="127.0.0.1",
                   MASTER_PORT=str(port))
        procs.append(subprocess.Popen([sys.executable, str(script)], env=env, stdout=subprocess.PIPE,
                                      stderr=subprocess.STDOUT, text=True))
    outs = []
    for p in procs:
        try:
            out, _ = p.communicate(timeout=120)
        except subprocess.TimeoutExpired:
            p.kill()
            out, _ = p.communicate()
        outs.append(out)
        assert p.returncode == 0, out
    assert "rank 0 ok" in outs[0] and "rank 1 ok" in outs[1]
