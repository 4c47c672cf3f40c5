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


SHARD_WORKER = r"""
import json, sys, datetime
sys.path.insert(0, sys.argv[1])
import numpy as np
import torch.distributed as dist
from mwa_hyperdrive_b200 import shard, synth
from oracle import oracle as O
dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=60))
rank, world = dist.get_rank(), dist.get_world_size()
rng = np.random.default_rng(3)
ntiles, nt, nch = 8, 2, 7
nbl = ntiles * (ntiles - 1) // 2
model = synth.random_model(nt, nch, nbl, rng)
data = synth.corrupt(model, synth.truth_gains(ntiles, nch, rng), rng, 30.0)
start = np.zeros((ntiles, nch, 8)); start[..., 0] = start[..., 6] = 1.0
start[:, 3] = 0.0; start[:, 4] = 0.0          # a run of failures across the shard edge
start[:, 0] = 0.0                             # a leading failure
c0, c1 = shard.ranges(nch, world)[rank]
d, m = data[:, c0:c1], model[:, c0:c1]
def solver(lst, starts):
    out = starts.copy(); res = [dict(converged=False)] * (c1 - c0)
    res = list(res)
    for k in (range(c1 - c0) if lst is None else lst):
        dj, r = O.calibrate(d, m, k, starts[:, k], 50, 1e-8, 1e-4, 0)
        out[:, k] = dj
        res[k] = dict(converged=bool(r.converged), num_iterations=r.num_iterations)
    return out, res
sols, res = shard.calibrate_timeblock_sharded(solver, start[:, c0:c1].copy(), c0, nch)
full = shard.gather_channels(np.moveaxis(sols, 1, 0), axis=0)
its = [r["num_iterations"] for r in res]
allits = [None] * world
dist.all_gather_object(allits, its)
if rank == 0:
    ref, rres = O.calibrate_timeblock(data, model, start, 0, nt, 50, 1e-8, 1e-4, 0)
    ok_nan = bool(np.array_equal(np.isnan(np.moveaxis(full, 0, 1)), np.isnan(ref)))
    fin = np.isfinite(ref)
    err = float(np.max(np.abs(np.moveaxis(full, 0, 1)[fin] - ref[fin]))) if fin.any() else 0.0
    print(json.dumps({"nan_equal": ok_nan, "err": err, "its": sum(allits, []),
                      "ref_its": [r["num_iterations"] for r in rres],
                      "converged": int(sum(r["converged"] for r in rres))}), flush=True)
dist.destroy_process_group()
"""


def test_sharded_calibration_equals_single_rank():
    """DI calibration with its chanblocks spread over 2 CPU ranks (the
    oracle's per-chanblock solver standing in for each GPU): the band-wide
    retry of failed chanblocks -- a run of failures across the shard edge and
    a leading one -- gives the single-process calibrate_timeblock's
    solutions, NaN pattern and iteration counts exactly."""
    outs = run_ranks(SHARD_WORKER, 2)
    line = [json.loads(o.strip().splitlines()[-1]) for o in outs if o.strip()][0]
    assert line["nan_equal"] and line["err"] == 0.0, line
    assert line["its"] == line["ref_its"], line
    assert line["converged"] == 7, line


GATHER_WORKER = r"""
import json, sys, datetime
sys.path.insert(0, sys.argv[1])
import numpy as np
import torch.distributed as dist
from mwa_hyperdrive_b200 import shard, synth
from oracle import oracle as O
dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=60))
rank, world = dist.get_rank(), dist.get_world_size()
obs, sky = synth.config1()
f0, f1 = shard.ranges(obs.freqs.size, world)[rank]
vis, _ = O.model_timestep(sky, obs.tile_xyzs[:20], obs.freqs[f0:f1], obs.phase_centre, obs.lsts[0], obs.latitude,
                          out_f64=True)
full = shard.gather_channels(vis, axis=0)
if rank == 0:
    ref, _ = O.model_timestep(sky, obs.tile_xyzs[:20], obs.freqs, obs.phase_centre, obs.lsts[0], obs.latitude,
                              out_f64=True)
    print(json.dumps({"equal": bool(np.array_equal(full, ref)), "shape": list(full.shape)}), flush=True)
dist.destroy_process_group()
"""


def test_channel_sharded_predict_gathers_the_band():
    outs = run_ranks(GATHER_WORKER, 3)
    line = [json.loads(o.strip().splitlines()[-1]) for o in outs if o.strip()][0]
    assert line["equal"] and line["shape"] == [32, 190, 8], line


def test_ranges_cover_the_band():
    from mwa_hyperdrive_b200 import shard

    for n, w in [(768, 8), (7, 2), (5, 8), (384, 3)]:
        r = shard.ranges(n, w)
        assert r[0][0] == 0 and r[-1][1] == n and all(a[1] == b[0] for a, b in zip(r, r[1:]))
        assert max(h - l for l, h in r) - min(h - l for l, h in r) <= 1
