"""The replica bookkeeping of bench.py on two gloo ranks (CPU, no GPU).

The path does not shard; under torchrun every rank runs its own replica and
the job's time is the maximum over ranks.  The reference arm runs on rank 0
only; the other ranks exit without work.
"""
import json
import os
import socket
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

WORKER = r"""
import os, sys, json
sys.path.insert(0, os.environ["ROOT"])
import torch.distributed as dist
from datetime import timedelta
import bench
rank = int(os.environ["RANK"])
dist.init_process_group("gloo", timeout=timedelta(seconds=60))
m = bench.max_over_ranks(1.5 + rank, device="cpu")
assert m == 1.5 + int(os.environ["WORLD_SIZE"]) - 1, m
# the reference arm: rank 0 alone does work (it is skipped here with --steps 0
# on rank 0 by not calling it); other ranks return at once
if rank != 0:
    assert bench.run_reference_arm(None, rank) is None
dist.barrier()
dist.destroy_process_group()
print(json.dumps({"rank": rank, "max": m}))
"""


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


@pytest.mark.timeout(180)
def test_max_over_ranks_and_reference_arm_on_two_gloo_ranks():
    port = _free_port()
    procs = []
    for r in range(2):
        env = dict(os.environ, ROOT=ROOT, RANK=str(r), LOCAL_RANK=str(r), WORLD_SIZE="2",
                   MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
        procs.append(subprocess.Popen([sys.executable, "-c", WORKER], env=env,
                                      stdout=subprocess.PIPE, stderr=subprocess.PIPE,
                                      text=True))
    outs = []
    for p in procs:
        out, err = p.communicate(timeout=170)
        assert p.returncode == 0, err[-2000:]
        outs.append(json.loads(out.strip().splitlines()[-1]))
    assert sorted(o["rank"] for o in outs) == [0, 1]
    assert all(o["max"] == 2.5 for o in outs)


def test_max_over_ranks_without_a_group_is_identity():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.max_over_ranks(3.25, device="cpu") == 3.25
