"""The bench's N-GPU path (independent replicas, weak scaling) on CPU ranks:
two gloo processes time different amounts of work; every rank must see the
maximum over ranks, the aggregate counts every rank's units, and under the
reference arm only rank 0 prints."""

import json
import os
import socket
import subprocess
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]

WORKER = r"""
import json, os, sys, datetime
sys.path.insert(0, sys.argv[1])
import torch.distributed as dist
import bench
dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=60))
rank, world = dist.get_rank(), dist.get_world_size()
t = bench.max_over_ranks(0.5 + rank, dist)          # rank r took 0.5 + r seconds
dist.barrier()
print(json.dumps({"rank": rank, "max": t, "value": bench.aggregate(100.0, world, t)}), flush=True)
dist.destroy_process_group()
"""


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def run_ranks(code, world, extra_args=()):
    port = free_port()
    procs = []
    for r in range(world):
        env = dict(os.environ, RANK=str(r), WORLD_SIZE=str(world), LOCAL_RANK=str(r), MASTER_ADDR="127.0.0.1",
                   MASTER_PORT=str(port), CUDA_VISIBLE_DEVICES="")
        procs.append(subprocess.Popen([sys.executable, "-c", code, str(ROOT), *extra_args], env=env,
                                      stdout=subprocess.PIPE, stderr=subprocess.PIPE, text=True))
    outs = []
    for p in procs:
        out, err = p.communicate(timeout=120)
        assert p.returncode == 0, err
        outs.append(out)
    return outs


def test_max_over_ranks_and_weak_aggregate():
    outs = run_ranks(WORKER, 2)
    lines = [json.loads(o.strip().splitlines()[-1]) for o in outs]
    assert sorted(l["rank"] for l in lines) == [0, 1]
    for l in lines:
        assert l["max"] == pytest.approx(1.5)
        assert l["value"] == pytest.approx(100.0 * 2 / 1.5)


def test_reference_arm_prints_on_rank_zero_only():
    code = r"""
import sys
sys.path.insert(0, sys.argv[1])
import bench
class A: pass
a = A(); a.steps = 1; a.warmup = 0; a.gpus = 2
bench.reference_arm(a, 1)   # a non-zero rank returns without work or output
print("done")
"""
    env = dict(os.environ, CUDA_VISIBLE_DEVICES="")
    out = subprocess.run([sys.executable, "-c", code, str(ROOT)], env=env, capture_output=True, text=True,
                         timeout=120)
    assert out.returncode == 0, out.stderr
    assert out.stdout.strip() == "done"
