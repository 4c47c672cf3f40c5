"""Benchmark: sky-model predict throughput (vis x components / s) on the
mixed-component configuration (128 tiles, 4 timesteps, 384 channels, 4000
points + 500 Gaussians + 100 shapelets, analytic beam), synthetic seeded
inputs.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

A step predicts all 4 timesteps of the configuration.  `value` is the
device-resident throughput (inputs and tables in HBM, L2 flushed between
steps, CUDA events on the launching stream, max over ranks); `e2e` is the
same metric through the trait-style C-ABI call with host buffers (H2D of the
accumulated visibilities and D2H of the result inside the timed region).
Multi-GPU runs are independent replicas (the predict shards by timestep and
channel with no exchange), so scaling is weak.

Rank 0 of a 1-GPU run adds sections measured the same way: `dical` (DI
calibration, all solver forms), `peel` (sequential and batched peeling),
`warmstart` (learned warm start against identity starts), `prep`
(vis_average and scale_by_weights against the HBM copy bandwidth) and `fee`
(the FEE beam's per-tile Jones against the FP64 FMA rate).
"""

from __future__ import annotations

import argparse
import ctypes
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "predict vis·components/s"
UNIT = "vis·comp/s"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="hdc", choices=["hdc", "reference"])
    ap.add_argument("--form", default="auto", choices=["auto", "direct", "tensor"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cpu-seconds", type=float, default=12.0)
    ap.add_argument("--channels", type=int, default=384, help="reduced case for profiling (default: full 384)")
    ap.add_argument("--timesteps", type=int, default=4, help="reduced case for profiling (default: full 4)")
    ap.add_argument("--skip-e2e", action="store_true")
    ap.add_argument("--skip-dical", action="store_true", help="leave out the DI-calibration measurement")
    ap.add_argument("--dical-chanblocks", type=int, default=768, help="reduced DI-cal case for profiling")
    ap.add_argument("--skip-peel", action="store_true", help="leave out the peeling measurement")
    ap.add_argument("--warm-chanblocks", type=int, default=768, help="reduced warm-start case for profiling")
    ap.add_argument("--skip-warmstart", action="store_true", help="leave out the warm-start measurement")
    ap.add_argument("--peel-channels", type=int, default=384, help="reduced peel case for profiling")
    ap.add_argument("--skip-prep", action="store_true", help="leave out the visibility-preparation measurement")
    ap.add_argument("--prep-timesteps", type=int, default=8, help="reduced visibility-preparation case for profiling")
    ap.add_argument("--skip-fee", action="store_true", help="leave out the FEE beam measurement")
    ap.add_argument("--fee-directions", type=int, default=4600, help="reduced FEE case for profiling")
    args = ap.parse_args()
    global SHAPE
    SHAPE = (args.channels, args.timesteps)
    return args


SHAPE = (384, 4)


def workload():
    from mwa_hyperdrive_b200 import synth

    obs, sky = synth.config2(n_freqs=SHAPE[0], n_times=SHAPE[1])
    return obs, sky


def vis_comp_per_step(obs, sky):
    return obs.num_baselines * obs.freqs.size * obs.lsts.size * sky.num_components


def config_dict(obs, sky, form):
    return {
        "workload": "mixed-component predict: 128 tiles (8128 baselines), 4 timesteps x 8 s, 384 x 80 kHz channels "
                    "from 167 MHz, 4000 points + 500 Gaussians + 100 shapelets (20 coeffs), curved power laws, "
                    "analytic dipole-array beam",
        "tiles": int(obs.num_tiles), "baselines": int(obs.num_baselines), "timesteps": int(obs.lsts.size),
        "channels": int(obs.freqs.size), "components": int(sky.num_components),
        "points": int(np.sum(sky.comp_type == 0)), "gaussians": int(np.sum(sky.comp_type == 1)),
        "shapelets": int(np.sum(sky.comp_type == 2)), "form": form,
        "l2": "flushed between steps (256 MiB write)",
    }


# ------------------------------------------------------------ replicas
def max_over_ranks(value: float, dist) -> float:
    """The largest of every rank's value (a time), on every rank; NCCL ranks
    reduce on their GPU, gloo ranks on the CPU."""
    if dist is None:
        return value
    import torch

    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([value], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def aggregate(work_per_rank: float, world: int, seconds_max: float) -> float:
    """Whole-job throughput of `world` independent replicas (weak scaling):
    every rank processed `work_per_rank` units, the slowest took seconds_max."""
    return work_per_rank * world / seconds_max


# ----------------------------------------------------------------- clocks
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.path = None

    def start(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"], stdout=self.f,
                                         stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        out = {"sm_mhz": None, "sm_max_mhz": None, "reasons": []}
        if self.proc is None:
            return out
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.f.close()
        rows = []
        for line in Path(self.path).read_text().splitlines():
            parts = [p.strip() for p in line.split(",")]
            if len(parts) >= 9:
                rows.append(parts)
        os.unlink(self.path)
        if not rows:
            return out
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        reasons = set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            for k, n in enumerate(names):
                if r[5 + k].lower() == "active":
                    reasons.add(n)
        out["sm_mhz"] = statistics.median(sm) if sm else None
        out["sm_max_mhz"] = max(mx) if mx else None
        out["reasons"] = sorted(reasons)
        out["samples"] = len(rows)
        return out


# --------------------------------------------------------- reference arm
def oracle_predict_samples(obs, sky, sample_s: float, samples: int):
    """The reference's CPU predictor (the oracle's C++ restatement of
    SkyModellerCpu, OpenMP over baselines, all host threads) timed on bounded
    samples of the workload: each sample is one timestep (cycling through the
    workload's) x the first nch channels, nch sized after a warm-up so that a
    sample takes about sample_s.  The cpu_baseline leg and the reference arm
    both use this one rule.  Returns (work per sample, seconds per sample
    list, nch, threads)."""
    from oracle import oracle as orc

    orc.build()
    threads = os.cpu_count() or 1
    orc.set_num_threads(threads)
    beam = orc.beam_struct(1)
    orc.model_timestep(sky, obs.tile_xyzs, obs.freqs[:1], obs.phase_centre, obs.lsts[0], obs.latitude, beam=beam)
    t0 = time.perf_counter()
    orc.model_timestep(sky, obs.tile_xyzs, obs.freqs[:2], obs.phase_centre, obs.lsts[0], obs.latitude, beam=beam)
    per_ch = (time.perf_counter() - t0) / 2
    nch = int(max(1, min(obs.freqs.size, round(sample_s / max(per_ch, 1e-4)))))
    times = []
    for k in range(samples):
        t0 = time.perf_counter()
        orc.model_timestep(sky, obs.tile_xyzs, obs.freqs[:nch], obs.phase_centre, obs.lsts[k % obs.lsts.size],
                           obs.latitude, beam=beam)
        times.append(time.perf_counter() - t0)
    return obs.num_baselines * nch * sky.num_components, times, nch, threads


def reference_arm(args, rank):
    """The reference's CPU predictor on bounded samples of the same workload
    (oracle_predict_samples: one step = one sample of ~3 s)."""
    if rank != 0:
        return
    obs, sky = workload()
    from oracle import oracle as orc

    orc.build()
    orc.set_num_threads(os.cpu_count() or 1)
    beam = orc.beam_struct(1)
    for _ in range(max(args.warmup, 0)):
        orc.model_timestep(sky, obs.tile_xyzs, obs.freqs[:1], obs.phase_centre, obs.lsts[0], obs.latitude, beam=beam)
    work, times, nch, threads = oracle_predict_samples(obs, sky, 3.0, max(args.steps, 1))
    value = work * len(times) / sum(times)
    sample = (f"per step: 1 timestep (cycling over the 4) x {nch} of {obs.freqs.size} channels x "
              f"{sky.num_components} components x {obs.num_baselines} baselines")
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": len(times), "warmup": args.warmup, "ms_per_step": 1e3 * sum(times) / len(times),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": config_dict(obs, sky, "reference CPU (C++ restatement of SkyModellerCpu, OpenMP)"),
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port", "sample": sample},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def cpu_baseline(obs, sky, seconds):
    """The same rule as the reference arm: samples of ~3 s, as many as fit in
    `seconds` (at least 4, one per timestep)."""
    samples = max(4, int(round(seconds / 3.0)))
    work, times, nch, threads = oracle_predict_samples(obs, sky, 3.0, samples)
    return {"value": work * len(times) / sum(times), "unit": UNIT, "cores": threads, "kind": "port",
            "sample": f"{len(times)} samples of 1 timestep (cycling over the 4) x {nch} of {obs.freqs.size} channels x "
                      f"{sky.num_components} components x {obs.num_baselines} baselines ({sum(times):.1f} s)"}


def sampled_error(vis_tfb, obs, sky, ntiles_sample=24, seed=2024):
    """Parity check of the timed output (the checker, run with the
    cpu_baseline leg): the chosen form's visibilities [t][f][bl][8] of every
    timestep and channel on a seeded sample of baselines (all baselines among
    ntiles_sample random tiles) against the FP64 oracle; normwise error and
    the 99.9th percentile of |dV| over the rms visibility."""
    import torch

    from mwa_hyperdrive_b200 import synth
    from oracle import oracle as orc

    orc.build()
    orc.set_num_threads(os.cpu_count() or 1)
    sub, bl = synth.sample_tiles(obs.num_tiles, ntiles_sample, seed)
    got = vis_tfb.index_select(2, torch.from_numpy(bl).to(vis_tfb.device)).cpu().numpy().astype(np.float64)
    t0 = time.perf_counter()
    ref = np.stack([orc.model_timestep(sky, obs.tile_xyzs[sub], obs.freqs, obs.phase_centre, float(lst), obs.latitude,
                                       beam=orc.beam_struct(1), out_f64=True)[0] for lst in obs.lsts])
    norm = np.linalg.norm(ref)
    rms = norm / math.sqrt(ref.size)
    d = np.abs(got - ref)
    return {"normwise": float(np.linalg.norm(got - ref) / norm), "p999": float(np.percentile(d, 99.9) / rms),
            "max": float(d.max() / rms), "bar": 1e-6, "vs": "FP64 oracle (C++ restatement of SkyModellerCpu)",
            "sample": f"{bl.size} baselines (all among {ntiles_sample} seeded random tiles) x {obs.freqs.size} channels "
                      f"x {obs.lsts.size} timesteps of the last timed step's output ({time.perf_counter() - t0:.1f} s)"}


# ------------------------------------- reference GPU kernels (baseline leg)
def dropin_inputs(obs, sky, lst, keep):
    """The reference FFI's device inputs (gpu/types.h Points / Gaussians /
    Shapelets / Addresses, FP64 build) for the workload's sky at one
    timestep: components grouped power law / curved power law per type,
    instrumental flux at 150 MHz, per-baseline UVWs and shapelet UVs, the
    shapelet basis table, and a beam of one unique tile and frequency (random
    Jones near identity: the same work per component as any beam)."""
    import torch

    from mwa_hyperdrive_b200 import _lib

    def put(a, dt=np.float64):
        t = torch.from_numpy(np.ascontiguousarray(a, dt)).cuda()
        keep.append(t)
        return t.data_ptr()

    pc = obs.phase_centre
    xyz = obs.tile_xyzs
    i, j = np.triu_indices(obs.num_tiles, 1)
    d = xyz[i] - xyz[j]

    def uvw(ha, dec):
        sh, ch, sd, cd = np.sin(ha), np.cos(ha), np.sin(dec), np.cos(dec)
        return np.stack([sh * d[:, 0] + ch * d[:, 1], -sd * ch * d[:, 0] + sd * sh * d[:, 1] + cd * d[:, 2],
                         cd * ch * d[:, 0] - cd * sh * d[:, 1] + sd * d[:, 2]], -1)

    nbl, nf = obs.num_baselines, obs.freqs.size
    sbf = np.zeros(101 * 10001)
    _lib.lib().hdc_shapelet_basis(sbf.ctypes.data)
    addr = _lib.Addresses(nf, nf * nbl, nbl, put(obs.freqs), put(sbf), 1, put(np.zeros(obs.num_tiles), np.int32),
                          put(np.zeros(nf), np.int32), put(np.arange(obs.num_tiles), np.int32))
    structs = {}
    coeff_dt = np.dtype([("value", np.float64), ("n1", np.uint8), ("n2", np.uint8), ("pad", np.uint8, 6)])
    rng = np.random.default_rng(9)
    for ct in range(3):
        idx = np.nonzero(sky.comp_type == ct)[0]
        groups = [idx[sky.flux_type[idx] == 1], idx[sky.flux_type[idx] == 2]]
        assert len(groups[0]) + len(groups[1]) == len(idx), "list fluxes are not part of this workload"
        order = np.concatenate(groups)
        nc = order.size
        ra, dec = sky.ra[order], sky.dec[order]
        dra = ra - pc[0]
        l = np.cos(dec) * np.sin(dra)
        m = np.sin(dec) * np.cos(pc[1]) - np.cos(dec) * np.sin(pc[1]) * np.cos(dra)
        n = np.sin(dec) * np.sin(pc[1]) + np.cos(dec) * np.cos(pc[1]) * np.cos(dra)
        lmn = 2 * np.pi * np.stack([l, m, n - 1.0], -1)
        fd = sky.fds[sky.fd_start[order]]
        assert np.all(fd[:, 0] == 150e6)
        # to_inst_stokes (srclist/types/flux_density/mod.rs:58-65): XX = I - Q,
        # XY = U - iV, YX = U + iV, YY = I + Q
        inst = np.zeros((nc, 8))
        inst[:, 0] = fd[:, 1] - fd[:, 2]
        inst[:, 2], inst[:, 3] = fd[:, 3], -fd[:, 4]
        inst[:, 4], inst[:, 5] = fd[:, 3], fd[:, 4]
        inst[:, 6] = fd[:, 1] + fd[:, 2]
        beam = rng.normal(size=(1, 1, nc, 8)) * 0.05
        beam[..., 0] += 1.0
        beam[..., 6] += 1.0
        n0 = groups[0].size
        lm, fdp, sis = put(lmn), put(inst), put(sky.si[order])
        qs = put(np.concatenate([sky.q[groups[1]], [0.0]]))
        if ct == 0:
            st = _lib.Points(n0, lm, fdp, sis, nc - n0, lm + 24 * n0, fdp + 64 * n0, sis + 8 * n0, qs, 0, 0, 0)
        else:
            gp = put(np.stack([sky.maj[order], sky.min[order], sky.pa[order]], -1))
        if ct == 1:
            st = _lib.Gaussians(n0, lm, fdp, sis, gp, nc - n0, lm + 24 * n0, fdp + 64 * n0, sis + 8 * n0, qs,
                                gp + 24 * n0, 0, 0, 0, 0)
        if ct == 2:
            suv = np.stack([uvw(lst - ra[k], dec[k])[:, :2] for k in range(nc)], 1)  # [bl][nc][2]
            cnt = sky.coeff_count[order]
            co = np.zeros(int(cnt.sum()), coeff_dt)
            pos = 0
            for k in order:
                a, b = sky.coeff_start[k], sky.coeff_start[k] + sky.coeff_count[k]
                co["value"][pos:pos + b - a] = sky.coeff_value[a:b]
                co["n1"][pos:pos + b - a] = sky.coeff_n1[a:b]
                co["n2"][pos:pos + b - a] = sky.coeff_n2[a:b]
                pos += b - a
            c0 = int(cnt[:n0].sum())
            suv_p = [put(suv[:, :n0]), put(suv[:, n0:])]
            cop, ncp = put(co.view(np.uint8), np.uint8), put(cnt, np.int32)
            st = _lib.Shapelets(n0, lm, fdp, sis, gp, suv_p[0], cop, ncp,
                                nc - n0, lm + 24 * n0, fdp + 64 * n0, sis + 8 * n0, qs, gp + 24 * n0, suv_p[1],
                                cop + 16 * c0, ncp + 4 * n0, 0, 0, 0, 0, 0, 0, 0)
        structs[ct] = (st, put(beam))
    return structs, addr, put(uvw(lst - pc[0], pc[1]))


def reference_gpu_leg(obs, sky):
    """Baseline leg: mwa_hyperdrive's own GPU kernels (src/gpu/model.cu, FP64
    build, compiled for sm_100a from the reference's sources into
    oracle/_ref/libref_gpu.so) against libhdc's drop-in kernels on identical
    device inputs, one timestep of the workload, CUDA events on the legacy
    default stream both libraries launch on, best of 3 after a warm-up.  The
    drop-in calls include their per-call table preparation and the read of
    their kernel error word."""
    import torch

    from mwa_hyperdrive_b200 import _lib

    so = ROOT / "oracle" / "_ref" / "libref_gpu.so"
    if not so.exists():
        return {"unavailable": "oracle/_ref/libref_gpu.so was not built (needs the reference sources)"}
    ref = ctypes.CDLL(str(so))
    names = {0: "model_points", 1: "model_gaussians", 2: "model_shapelets"}
    for nm in names.values():
        res, argt = _lib.SIGNATURES[nm]
        getattr(ref, nm).restype, getattr(ref, nm).argtypes = res, argt
    keep = []
    structs, addr, uvws = dropin_inputs(obs, sky, float(obs.lsts[0]), keep)
    nf, nbl = obs.freqs.size, obs.num_baselines
    out = {"workload": "one timestep of the mixed-component workload (4000 points, 500 Gaussians, 100 shapelets, "
                       "384 channels, 8128 baselines) through the reference FFI with a per-tile beam table of one "
                       "unique tile", "unit": "ms per timestep"}
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
    vis = {k: torch.zeros((nf, nbl, 8), dtype=torch.float32, device="cuda") for k in ("ref", "hdc")}
    total = {"ref": 0.0, "hdc": 0.0}
    for ct, nm in names.items():
        st, beam = structs[ct]
        row = {}
        for who, lib in (("ref", ref), ("hdc", _lib.lib())):
            fn = getattr(lib, nm)
            best = float("inf")
            for rep in range(4):
                vis[who].zero_()
                torch.cuda.synchronize()
                ev[0].record(torch.cuda.default_stream())
                _lib.check_str(fn(ctypes.byref(st), ctypes.byref(addr), uvws, beam, vis[who].data_ptr()),
                               f"{who} {nm}")
                ev[1].record(torch.cuda.default_stream())
                torch.cuda.synchronize()
                if rep:
                    best = min(best, ev[0].elapsed_time(ev[1]))
            row[who + "_ms"] = best
            total[who] += best
        a, b = vis["hdc"].double(), vis["ref"].double()
        row["max_abs_diff_over_rms"] = float((a - b).abs().max() / b.pow(2).mean().sqrt())
        row["speedup"] = row["ref_ms"] / row["hdc_ms"]
        out[nm] = row
    out["all_types"] = {"ref_ms": total["ref"], "hdc_ms": total["hdc"], "speedup": total["ref"] / total["hdc"]}
    del keep
    return out


# ------------------------------------------------------ DI calibration
DICAL_WORKLOAD = ("DI calibration: 128 tiles (8128 baselines), 1 timeblock of 14 timesteps 8 s apart, 768 chanblocks "
                  "of 40 kHz from 167 MHz; truth gains |g| ~ N(1, 0.1), phase U(-pi, pi), leakage N(0, 0.01); model "
                  "predicted from 8000 points (lognormal(0, 1) Jy, 10 deg cap) through the analytic dipole-array beam "
                  "(an unpolarised sky without a beam gives M proportional to I, for which full-Jones solutions are "
                  "defined only up to a unitary factor and no chanblock converges); data = G M G^H + noise at "
                  "per-visibility SNR 10; max 50 iterations, stop 1e-8, min 1e-4")


def dical_workload(nch):
    """Model and data [14][nch][8128][8] float32 on the device, and the truth gains."""
    import torch

    from mwa_hyperdrive_b200 import synth
    from mwa_hyperdrive_b200 import srclist as sl
    from mwa_hyperdrive_b200.model import SkyModeller

    pc = (0.0, math.radians(-27.0))
    nt = 14
    lsts = pc[0] + np.arange(nt) * 8.0 * synth.SIDEREAL_RATE
    obs = synth.Obs(synth.tiles_in_disk(128, 750.0, 3), 167.0e6 + np.arange(nch) * 40e3, pc, lsts)
    sky = sl.SkyModelArrays.from_components(synth.point_sky(8000, pc, 10.0, 3))
    nbl = obs.num_baselines
    model = torch.zeros((nt, nch, nbl, 8), dtype=torch.float32, device="cuda")
    m = SkyModeller(sky, obs.tile_xyzs, obs.freqs, pc, obs.latitude, beam="analytic", form="tensor")
    for t in range(nt):
        m.model_timestep_with(float(lsts[t]), model[t], return_uvws=False)
    m.close()
    rng = np.random.default_rng(3)
    g = synth.truth_gains(128, nch, rng)  # [tile][chanblock][8]
    gc = torch.from_numpy(g[..., 0::2] + 1j * g[..., 1::2]).to("cuda").reshape(128, nch, 2, 2)
    i, j = np.triu_indices(128, 1)
    ii, jj = torch.from_numpy(i).cuda(), torch.from_numpy(j).cuda()
    data = torch.empty_like(model)
    gen = torch.Generator(device="cuda")
    gen.manual_seed(3)
    for t in range(nt):
        mc = torch.view_as_complex(model[t].reshape(nch, nbl, 4, 2)).reshape(nch, nbl, 2, 2).to(torch.complex128)
        gp = gc[ii].permute(1, 0, 2, 3)  # [nch][nbl][2][2]
        gq = gc[jj].permute(1, 0, 2, 3)
        d = gp @ mc @ gq.conj().transpose(-1, -2)
        dr = torch.view_as_real(d.reshape(nch, nbl, 4)).reshape(nch, nbl, 8)
        rms = torch.sqrt(torch.mean(dr[..., [0, 1, 6, 7]] ** 2))
        noise = torch.randn(dr.shape, generator=gen, device="cuda", dtype=torch.float64) * (rms / 10.0 / math.sqrt(2.0))
        data[t] = (dr + noise).to(torch.float32)
    return model, data, g


def dical_arm(args):
    """DI calibration of the workload's timeblock in every solver form, each
    timed best of 3 (CUDA-synchronised wall time of the whole call: the CUDA
    graph of the first pass, the retry pass and the result reads).  Two
    budgets: the stated 50 iterations (on this sky no chanblock converges in
    50 iterations -- the CPU oracle agrees -- so every chanblock ends failed
    and NaN-padded, as the reference does) and 200 iterations, where the
    solver converges (mean ~130 iterations); the 200-iteration run is the
    headline and is checked against the CPU oracle on sampled chanblocks."""
    import torch

    from mwa_hyperdrive_b200 import calibrate as cal

    nch = args.dical_chanblocks
    model, data, g = dical_workload(nch)
    nt = model.shape[0]
    ident = np.zeros((128, nch, 8))
    ident[..., 0] = 1.0
    ident[..., 6] = 1.0
    out = {"workload": DICAL_WORKLOAD, "metric": "DI-cal s/timeblock", "unit": "s", "higher_is_better": False}
    forms = ("plain", "collapsed", "collapsed_f32")

    def run(max_iter):
        res_by_form, sols, its = {}, {}, {}
        for form in forms:
            dj = torch.from_numpy(ident.copy()).cuda()
            cal.calibrate_timeblock(data, model, dj, (0, nt), max_iter, 1e-8, 1e-4, form=form)  # warm-up
            times, res = [], None
            for _ in range(3):
                dj.copy_(torch.from_numpy(ident))
                torch.cuda.synchronize()
                t0 = time.perf_counter()
                res = cal.calibrate_timeblock(data, model, dj, (0, nt), max_iter, 1e-8, 1e-4, form=form)
                torch.cuda.synchronize()
                times.append(time.perf_counter() - t0)
            sols[form] = dj.cpu().numpy()
            it = np.array([r.num_iterations for r in res])
            its[form] = it
            res_by_form[form] = {"s_per_timeblock": min(times), "s_all_runs": times,
                                 "iterations_mean": float(it.mean()), "iterations_max": int(it.max()),
                                 "converged": int(sum(r.converged for r in res)), "chanblocks": nch,
                                 "failed_chanblocks": int(np.isnan(sols[form]).any(axis=(0, 2)).sum())}
        ok = np.isfinite(sols["plain"])
        for form in forms[1:]:
            a, b = sols[form][ok], sols["plain"][ok]
            res_by_form[form]["solution_rel_err_vs_plain"] = (float(np.linalg.norm(a - b) / np.linalg.norm(b))
                                                              if ok.any() else None)
            res_by_form[form]["nan_pattern_equal"] = bool(np.array_equal(np.isnan(sols[form]),
                                                                         np.isnan(sols["plain"])))
        return res_by_form, sols, its

    out["max50"], _, _ = run(50)
    out["max50"]["note"] = ("the stated budget: no chanblock of this sky converges within 50 iterations (the CPU "
                            "oracle agrees), so every solution is NaN-padded as the reference does; times kept for "
                            "the iteration cost")
    conv, sols, its = run(200)
    out["to_convergence_max200"] = conv
    out["chosen"] = "collapsed_f32"
    out["headline_s_per_timeblock"] = conv["collapsed_f32"]["s_per_timeblock"]
    out["speedup_chosen_vs_plain"] = conv["plain"]["s_per_timeblock"] / conv["collapsed_f32"]["s_per_timeblock"]
    nbl = model.shape[2]
    it_total = conv["collapsed_f32"]["iterations_mean"] * nch
    out["algorithmic"] = {"plain_bytes_per_iteration_per_chanblock": nt * nbl * 64,
                          "collapsed_f32_bytes_per_iteration_per_chanblock": nbl * 48 * 4,
                          "fp64_flop_per_visibility_iteration_plain": 368, "collapsed_iterations_total": it_total}
    if not args.no_cpu_baseline:
        # the reference's CPU solver (oracle restatement of calibrate_timeblock,
        # OpenMP over chanblocks as rayon) at the same 200-iteration budget on
        # a sample of chanblocks, scaled; and every GPU form's solutions on
        # those chanblocks against it (bar 1e-6; the plain form follows the
        # oracle's arithmetic and agrees to ~1e-10)
        from oracle import oracle as orc

        orc.build()
        threads = os.cpu_count() or 1
        orc.set_num_threads(threads)
        ns = min(nch, max(threads, 8))
        pick = np.linspace(0, nch - 1, ns).round().astype(int)
        dh = data[:, pick].cpu().numpy()
        mh = model[:, pick].cpu().numpy()
        t0 = time.perf_counter()
        dj_o, res_o = orc.calibrate_timeblock(dh, mh, ident[:, pick], 0, nt, 200, 1e-8, 1e-4, 0)
        dt = time.perf_counter() - t0
        out["cpu_baseline"] = {"value": dt * nch / ns, "unit": "s", "cores": threads, "kind": "port",
                               "max_iterations": 200,
                               "sample": f"{ns} of {nch} chanblocks (evenly spaced) x 14 timesteps x {nbl} baselines "
                                         f"in {dt:.2f} s, scaled to {nch} chanblocks"}
        out["cpu_baseline"]["iterations_mean"] = float(np.mean([r["num_iterations"] for r in res_o]))
        for form in forms:
            a = sols[form][:, pick]
            ok = np.isfinite(dj_o) & np.isfinite(a)
            conv[form]["solution_rel_err_vs_oracle"] = (float(np.linalg.norm(a[ok] - dj_o[ok]) /
                                                              np.linalg.norm(dj_o[ok])) if ok.any() else None)
            conv[form]["oracle_nan_pattern_equal"] = bool(np.array_equal(np.isnan(a), np.isnan(dj_o)))
            conv[form]["oracle_iterations_equal"] = bool(np.array_equal(its[form][pick],
                                                                        [r["num_iterations"] for r in res_o]))
        out["speedup_chosen_vs_cpu"] = out["cpu_baseline"]["value"] / conv["collapsed_f32"]["s_per_timeblock"]
    return out


# ------------------------------------------------------------- peeling
PEEL_WORKLOAD = ("peeling: 128 tiles (8128 baselines), 8 timesteps 8 s apart, 384 x 80 kHz channels from 167 MHz "
                 "averaged x16 to 24 for the fits; sky of 20000 points (lognormal(0, 1) Jy, 10 deg cap); the 50 "
                 "brightest carry ionospheric offsets (alpha, beta) ~ N(0, 2e-5) and gains U(0.9, 1.1); residual = "
                 "data - model without ionosphere (so only those 50 remain); 3 passes x 10 iono iterations, "
                 "convergence 1, no beam")


def peel_workload(nch, sigma=2e-5):
    """Residual [8][nch][8128][8] float32 on the device, the 50 sources,
    their positions and truths (offsets N(0, sigma))."""
    import torch

    from mwa_hyperdrive_b200 import synth
    from mwa_hyperdrive_b200 import srclist as sl
    from mwa_hyperdrive_b200.model import SkyModeller

    pc = (0.0, math.radians(-27.0))
    nt = 8
    lsts = pc[0] + np.arange(nt) * 8.0 * synth.SIDEREAL_RATE
    obs = synth.Obs(synth.tiles_in_disk(128, 750.0, 5), 167.0e6 + np.arange(nch) * 80e3, pc, lsts)
    comps = synth.point_sky(20000, pc, 10.0, 5)
    flux = np.array([c.flux_type.fd.i for c in comps])
    bright = np.argsort(flux)[::-1][:50]
    rng = np.random.default_rng(5)
    nbl = obs.num_baselines
    lam = torch.from_numpy(299792458.0 / obs.freqs).cuda()
    resid = torch.zeros((nt, nch, nbl, 8), dtype=torch.float32, device="cuda")
    sources, positions, truths = [], [], []
    i, j = np.triu_indices(128, 1)
    for k in bright:
        sky = sl.SkyModelArrays.from_components([comps[k]])
        pos = (comps[k].ra, comps[k].dec)
        tr = (float(rng.normal(0, sigma)), float(rng.normal(0, sigma)), float(rng.uniform(0.9, 1.1)))
        sources.append(sky)
        positions.append(pos)
        truths.append(tr)
        m = SkyModeller(sky, obs.tile_xyzs, obs.freqs, pc, obs.latitude, beam="none", form="direct")
        for t in range(nt):
            mv = torch.zeros((nch, nbl, 8), dtype=torch.float64, device="cuda")
            m.model_timestep_with(float(lsts[t]), mv, return_uvws=False)
            # baseline u, v in the source's frame
            ha, dec = lsts[t] - pos[0], pos[1]
            xyz = obs.tile_xyzs
            d = xyz[i] - xyz[j]
            u = np.sin(ha) * d[:, 0] + np.cos(ha) * d[:, 1]
            v = -np.sin(dec) * np.cos(ha) * d[:, 0] + np.sin(dec) * np.sin(ha) * d[:, 1] + np.cos(dec) * d[:, 2]
            arg = -2 * np.pi * (torch.from_numpy(u * tr[0] + v * tr[1]).cuda()[None, :] * lam[:, None])
            f = torch.polar(torch.full_like(arg, tr[2]), arg) - 1.0  # iono - 1
            mc = torch.view_as_complex(mv.reshape(nch, nbl, 4, 2))
            resid[t] += torch.view_as_real(mc * f[..., None]).reshape(nch, nbl, 8).to(torch.float32)
        m.close()
    return obs, resid, sources, positions, truths


def peel_arm(args):
    import torch

    from mwa_hyperdrive_b200 import peel as P

    nch = args.peel_channels
    obs, resid0, sources, positions, truths = peel_workload(nch)
    weights = torch.ones(resid0.shape[:3], dtype=torch.float32, device="cuda")
    avg = float(np.median(obs.lsts))
    out = {"workload": PEEL_WORKLOAD, "metric": "peel s/timeblock (3 passes, 50 sources)", "unit": "s",
           "higher_is_better": False}
    def run_arm(resid_in, truths_, batched, batch_size=0, reps=3):
        times, consts, r = [], None, None
        for rep in range(reps):  # the first run also builds the models and (batched) autotunes
            r = resid_in.clone()
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            consts = P.peel_timeblock(r, weights, obs.freqs, obs.tile_xyzs, obs.lsts, avg, obs.phase_centre, sources,
                                      positions, [P.IonoConsts() for _ in sources], 3, 10, 1.0, 16,
                                      obs.latitude, "none", batched=batched, batch_size=batch_size)
            torch.cuda.synchronize()
            times.append(time.perf_counter() - t0)
        err_a = [abs(c.alpha - t[0]) for c, t in zip(consts, truths_)]
        err_g = [abs(c.gain - t[2]) for c, t in zip(consts, truths_)]
        # a source is captured when its fitted offset is within 10 % of the
        # injected one (or 1e-7) and its gain within 1e-3
        cap = sum(1 for c, t in zip(consts, truths_)
                  if abs(c.alpha - t[0]) < 0.1 * abs(t[0]) + 1e-7 and abs(c.beta - t[1]) < 0.1 * abs(t[1]) + 1e-7
                  and abs(c.gain - t[2]) < 1e-3)
        return {"s_per_timeblock": min(times), "first_call_s": times[0],
                "residual_rms_ratio": float(r.norm() / resid_in.norm()),
                "max_alpha_err": max(err_a), "max_gain_err": max(err_g), "captured": cap, "sources": len(truths_)}

    out["sequential"] = run_arm(resid0, truths, False)
    out["batched"] = run_arm(resid0, truths, True)
    bx, sy, ms = P.batched_tuning()
    out["batched"]["autotuned_accumulate_cta"] = {"bins": bx, "sources": sy, "ms": ms}
    # sub-batches of 10 in the list's (brightness) order: Jacobi within, the
    # reference's Gauss-Seidel order between them
    out["batched_sub10"] = run_arm(resid0, truths, True, 10)
    out["speedup_batched_vs_sequential"] = out["sequential"]["s_per_timeblock"] / out["batched"]["s_per_timeblock"]
    out["speedup_batched_sub10_vs_sequential"] = (out["sequential"]["s_per_timeblock"] /
                                                  out["batched_sub10"]["s_per_timeblock"])
    # the stated offsets, N(0, 2e-4): the reference's linearised fit does not
    # capture every draw on this array (tests/test_iono_capture.py); count
    # the captured sources of each arm (one timed run each)
    # (same seed: the same sources and positions, other offset draws)
    _, resid2, _, _, truths2 = peel_workload(nch, 2e-4)
    del resid0
    torch.cuda.empty_cache()
    out["stated_offsets_2e-4"] = {"sequential": run_arm(resid2, truths2, False, reps=1),
                                  "batched": run_arm(resid2, truths2, True, reps=1),
                                  "batched_sub10": run_arm(resid2, truths2, True, 10, reps=1)}
    del resid2
    if not args.no_cpu_baseline:
        # the reference's CPU peel loop (oracle restatement of peel_cpu,
        # params/peel/mod.rs:1121-1475, its rayon loops over timesteps as
        # OpenMP) on a sample -- the first 32 channels (two fit channels of
        # 16) and the first 4 sources for 1 pass of 10 iono iterations --
        # scaled by channels x sources x passes (each source's pass does the
        # same work; its iono loop may stop early on a step below 1e-8)
        from oracle import oracle as orc

        orc.build()
        threads = os.cpu_count() or 1
        orc.set_num_threads(threads)
        ns, nchs = 4, 32
        r_h = peel_workload(nchs)[1].cpu().numpy()
        w_h = np.ones(r_h.shape[:3], np.float32)
        t0 = time.perf_counter()
        orc.peel_cpu(r_h, w_h, obs.freqs[:nchs], obs.tile_xyzs, obs.lsts, avg, obs.phase_centre, sources[:ns],
                     positions[:ns], [(0.0, 0.0, 1.0)] * ns, 1, 10, 1.0, 16, obs.latitude)
        dt = time.perf_counter() - t0
        scale = (len(sources) / ns) * 3 * (nch / nchs)
        out["cpu_baseline"] = {"value": dt * scale, "unit": "s", "cores": threads, "kind": "port",
                               "sample": f"{ns} of {len(sources)} sources x 1 of 3 passes x {nchs} of {nch} channels "
                                         f"in {dt:.2f} s, scaled by {scale:.0f}"}
        out["speedup_batched_vs_cpu"] = out["cpu_baseline"]["value"] / out["batched"]["s_per_timeblock"]
        out["speedup_sequential_vs_cpu"] = out["cpu_baseline"]["value"] / out["sequential"]["s_per_timeblock"]
    nvis = int(np.prod(weights.shape))
    out["algorithmic"] = {"hi_res_vis": nvis, "hi_res_bytes": nvis * 32,
                          "batched_hi_res_bytes_per_pass": "residual read + read/write, weights, 50 model reads x 2"}
    return out


# ---------------------------------------------------------- warm start
WARM_WORKLOAD = ("learned warm start: 128 tiles, 768 chanblocks of 40 kHz, 4 timesteps per timeblock (the mixed "
                 "configuration's timesteps); gains with per-tile phase slopes U(-0.5, 0.5) rad/MHz drifting by 0.15 MHz "
                 "of slope per timeblock, 0.05 % amplitude jitter, leakage N(0, 0.01), polarised random sky (drawn on "
                 "the device); network 40 -> 3 x 256 -> 8 trained on the GPU (15 epochs) from identity-start solutions "
                 "of one seeded 4-timeblock sequence (3 transitions x 768 chanblocks = 2304 calibration instances); "
                 "evaluated on 7 transitions of an unseen 8-timeblock sequence at three solver operating points, and on "
                 "an off-model sequence (slopes U(-1.5, 1.5) rad/MHz, 3x the drift); warm-start time includes the "
                 "device features, network, judge and solve")


def warmstart_arm(args):
    import torch

    from mwa_hyperdrive_b200 import warmstart as ws

    ntiles, nch, ntb = 128, args.warm_chanblocks, 4
    tight = (400, 1e-15)

    def solve_seq(blocks, mlp, max_it, stop):
        prev, sols, iters, secs, chose = None, [], [], [], []
        for data, model, _ in blocks:
            sol, res, use, dt = ws.calibrate_warm(data, model, (0, int(data.shape[0])), prev, mlp,
                                                  max_iterations=max_it, stop_threshold=stop, min_threshold=1e-4)
            sols.append(sol)
            iters.append(int(sum(r.num_iterations for r in res)))
            secs.append(dt)
            chose.append(float(use.float().mean()) if use is not None else 0.0)
            prev = sol
        return sols, iters, secs, chose

    def compare(blocks, mlp, max_it, stop):
        s_id, it_id, t_id, _ = solve_seq(blocks, None, max_it, stop)
        s_ws, it_ws, t_ws, chose = solve_seq(blocks, mlp, max_it, stop)
        errs, failed = [], 0
        for k in range(1, len(blocks)):
            a, b = ws.gauge_align(s_ws[k].cpu().numpy()), ws.gauge_align(s_id[k].cpu().numpy())
            ok = np.isfinite(a) & np.isfinite(b)
            errs.append(float(np.max(np.abs(a[ok] - b[ok])) / np.max(np.abs(b[ok]))) if ok.any() else float("nan"))
            failed += int(np.isnan(a).any(axis=(0, 2)).sum())
        return {"max_iterations": max_it, "stop_threshold": stop,
                "identity": {"s_per_timeblock": float(np.mean(t_id[1:])),
                             "iterations_per_timeblock": float(np.mean(it_id[1:]))},
                "warm": {"s_per_timeblock": float(np.mean(t_ws[1:])),
                         "iterations_per_timeblock": float(np.mean(it_ws[1:])),
                         "chanblocks_using_proposal": float(np.mean(chose[1:])), "failed_chanblocks": failed},
                "wall_time_ratio": float(np.mean(t_id[1:]) / np.mean(t_ws[1:])),
                "iteration_ratio": float(np.mean(it_id[1:]) / np.mean(it_ws[1:])),
                "max_solution_diff_rel": max(errs)}, s_ws

    t0 = time.perf_counter()
    blocks = ws.DriftSky(ntiles, nch, ntb, 4, seed=200).generate(device=True)
    sols, _, _, _ = solve_seq(blocks, None, *tight)
    X, Y = [], []
    for k in range(1, len(sols)):
        X.append(ws.features_device(sols[k - 1]))
        Y.append(torch.from_numpy(ws.targets(sols[k - 1].cpu().numpy(), sols[k].cpu().numpy())).cuda())
    del blocks
    X, Y = torch.cat(X), torch.cat(Y)
    ok = torch.isfinite(X).all(dim=1) & torch.isfinite(Y).all(dim=1)
    mlp = ws.WarmStartMLP(hidden=256, num_hidden=3, seed=0)
    t1 = time.perf_counter()
    losses = mlp.train(X[ok], Y[ok], epochs=15, batch=4096, lr=1e-3)
    torch.cuda.synchronize()
    train_s = time.perf_counter() - t1
    n_inst = (len(sols) - 1) * nch
    del X, Y
    out = {"workload": WARM_WORKLOAD, "metric": "DI-cal s/timeblock with the learned warm start vs identity start",
           "unit": "s", "higher_is_better": False, "chanblocks": nch, "training_instances": n_inst,
           "train_s": train_s, "train_loss_first_last": [losses[0], losses[-1]]}
    blocks = ws.DriftSky(ntiles, nch, ntb, 8, seed=999).generate(device=True)
    solve_seq(blocks[:2], mlp, *tight)  # warm-up of both paths
    ops = {"stop1e-15_max400": tight, "stop1e-8_max50": (50, 1e-8), "stop1e-8_max200": (200, 1e-8)}
    for name, (max_it, stop) in ops.items():
        out[name], s_last = compare(blocks, mlp, max_it, stop)
    out["headline"] = "stop1e-15_max400"
    # the CPU arm: the reference's solver (oracle restatement of
    # calibrate_timeblock, OpenMP over chanblocks) on 16 evenly spaced
    # chanblocks of the last evaluated transition, from identity and from the
    # device chain's judged start, at stop 1e-8 / max 200; scaled to 768
    if not args.no_cpu_baseline:
        from oracle import oracle as orc

        orc.build()
        threads = os.cpu_count() or 1
        orc.set_num_threads(threads)
        data, model, _ = blocks[-1]
        prev = solve_seq(blocks[:-1], mlp, 200, 1e-8)[0][-1]
        start, _ = mlp.propose_device(prev, data, model, (0, int(data.shape[0])))
        pick = np.linspace(0, nch - 1, 16).round().astype(int)
        dh, mh = data[:, pick].cpu().numpy(), model[:, pick].cpu().numpy()
        res_cpu = {}
        for arm, s0 in (("identity", ws.identity_gains(ntiles, pick.size)), ("warm", start[:, pick].cpu().numpy())):
            t2 = time.perf_counter()
            _, r = orc.calibrate_timeblock(dh, mh, s0, 0, ntb, 200, 1e-8, 1e-4, 0)
            dt = time.perf_counter() - t2
            res_cpu[arm] = {"s_per_timeblock": dt * nch / pick.size,
                            "iterations_mean": float(np.mean([x["num_iterations"] for x in r]))}
        out["cpu_baseline"] = {"value": res_cpu["identity"]["s_per_timeblock"], "unit": "s", "cores": threads,
                               "kind": "port", "identity": res_cpu["identity"], "warm": res_cpu["warm"],
                               "wall_time_ratio": res_cpu["identity"]["s_per_timeblock"] /
                               res_cpu["warm"]["s_per_timeblock"],
                               "sample": f"16 of {nch} chanblocks (evenly spaced) of one transition, stop 1e-8, max "
                                         f"200, scaled to {nch}"}
    del blocks
    # a sequence the network was not trained for: three times wider slopes and
    # three times the drift; the judge must fall back where the proposal is worse
    off = ws.DriftSky(ntiles, nch, ntb, 8, seed=4242, slope_rad_per_mhz=1.5, drift_per_block=0.45).generate(device=True)
    out["off_model_stop1e-8_max200"], _ = compare(off, mlp, 200, 1e-8)
    del off
    out["data_and_training_s"] = time.perf_counter() - t0
    return out


# ----------------------------------------------- visibility preparation
PREP_WORKLOAD = ("visibility preparation before DI calibration: vis_average of one timeblock of 8 timesteps x 1536 "
                 "channels of 20 kHz x 8128 baselines (128 tiles) into 744 chanblocks of 40 kHz (24 coarse-channel "
                 "centre chanblocks flagged), then scale_by_weights of data and model of 8 timesteps x 744 "
                 "chanblocks x 8128 baselines with per-baseline weights; 15 % of weights <= 0")


def prep_arm(args):
    import torch

    from mwa_hyperdrive_b200 import calibrate as C

    nt, nf, nbl, nout = args.prep_timesteps, 1536, 8128, 744
    flagged = list(range(16, 768, 32))
    g = torch.Generator(device="cuda").manual_seed(11)
    vis = torch.randn((nt, nf, nbl, 8), generator=g, device="cuda")
    w = torch.rand((nt, nf, nbl), generator=g, device="cuda") * 20.0 - 3.0
    peaks = json.loads((ROOT / "MEASURED_PEAKS.json").read_text()) if (ROOT / "MEASURED_PEAKS.json").exists() else {}
    hbm = peaks.get("hbm_gbs", 6650.0)
    out = {"workload": PREP_WORKLOAD, "unit": "GB/s"}
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]

    def timed(fn, reps=5):
        fn()
        best = float("inf")
        for _ in range(reps):
            torch.cuda.synchronize()
            ev[0].record()
            fn()
            ev[1].record()
            torch.cuda.synchronize()
            best = min(best, ev[0].elapsed_time(ev[1]) * 1e-3)
        return best

    # inputs (3.6 GB) exceed L2; each call reads them once
    t_avg = timed(lambda: C.vis_average(vis, w, nout, flagged))
    bytes_avg = nt * nout * 2 * nbl * 36 + nout * nbl * 36  # used channels read once, outputs written once
    out["vis_average"] = {"s": t_avg, "algorithmic_bytes": bytes_avg, "achieved_gbs": bytes_avg / t_avg / 1e9,
                          "peak_gbs": hbm, "frac": bytes_avg / t_avg / 1e9 / hbm}
    del vis, w
    torch.cuda.empty_cache()
    d = torch.randn((nt, nout, nbl, 8), generator=g, device="cuda")
    m = torch.randn((nt, nout, nbl, 8), generator=g, device="cuda")
    wt = torch.rand((nt, nout, nbl), generator=g, device="cuda") * 20.0 - 3.0
    bw = np.linspace(0.0, 1.0, nbl)
    # count what scale_kernel moves: the weight of every entry, data and model
    # read only where weight x baseline weight > 0 (elsewhere zeros are
    # stored without a read), data and model written everywhere, and the
    # baseline weights (the weights are drawn once and not changed by the call)
    n_all = nt * nout * nbl
    n_pos = int(((wt.double() * torch.from_numpy(bw).cuda()[None, None, :]) > 0).sum())
    t_sc = timed(lambda: C.scale_by_weights(d, m, wt, bw))
    bytes_sc = n_all * 4 + n_pos * 2 * 32 + n_all * 2 * 32 + nbl * 8
    out["scale_by_weights"] = {"s": t_sc, "algorithmic_bytes": bytes_sc, "achieved_gbs": bytes_sc / t_sc / 1e9,
                               "peak_gbs": hbm, "frac": bytes_sc / t_sc / 1e9 / hbm}
    out["peak_source"] = "MEASURED_PEAKS.json hbm_gbs" if peaks else "fallback 6650 GB/s"
    if not args.no_cpu_baseline:
        from oracle import oracle as O

        O.build()
        rng = np.random.default_rng(2)
        sb = 1016  # a 1/8 sample of the baselines
        hv = rng.normal(size=(nt, nf, sb, 8)).astype(np.float32)
        hw = (rng.uniform(size=(nt, nf, sb)) * 20.0 - 3.0).astype(np.float32)
        t0 = time.perf_counter()
        O.vis_average(hv, hw, nout, flagged)
        dt = time.perf_counter() - t0
        out["cpu_baseline"] = {"value": dt * nbl / sb, "unit": "s per vis_average", "cores": 1, "kind": "port",
                               "sample": f"{sb} of {nbl} baselines, scaled by {nbl / sb:.1f}"}
        out["vis_average"]["speedup_vs_cpu"] = out["cpu_baseline"]["value"] / t_avg
    return out


FEE_NMAX = 16
FEE_WORKLOAD = ("FEE beam Jones (norm to zenith, parallactic rotation) at the mixed configuration's 4600 "
                "component directions for 128 tiles (24 unique: one pointing, 23 dead-dipole patterns) x 384 "
                "channels (their 25 closest file frequencies), synthetic coefficients with the beam file's "
                f"layout up to degree {FEE_NMAX} ({FEE_NMAX * (FEE_NMAX + 2)} modes per polarisation)")
FEE_FLOP_PER_MODE = 56  # both polarisations: theta and phi sums, 2 x (6 + 6 + 8 + 8)


def fee_arm(args):
    import torch

    from mwa_hyperdrive_b200 import _lib, synth
    from mwa_hyperdrive_b200.fee import FeeBeam

    lib = _lib.lib()
    file_f = (166.4e6 + np.arange(27) * 1.28e6).astype(np.uint32)
    coeffs = synth.fee_coeffs(file_f, FEE_NMAX, seed=21)
    chans = 167.00e6 + np.arange(384) * 0.08e6
    ntiles = 128
    base = np.array([(d % 4) * 3 + (d // 4) for d in range(16)], np.uint32)
    delays = np.tile(base, (ntiles, 1))
    for t in range(1, 24):  # tiles 1..23 each with its own dead dipole; the rest intact
        delays[t, (t * 5) % 16] = 32
        if t > 16:
            delays[t, (t * 3 + 1) % 16] = 32
    amps = np.ones((ntiles, 32))
    beam = FeeBeam(coeffs, chans, delays, amps, norm_to_zenith=True)
    nu, nuf = beam.num_unique_tiles(), beam.num_unique_freqs()
    n = args.fee_directions
    rng = np.random.default_rng(5)
    az = torch.from_numpy(rng.uniform(0.0, 2 * math.pi, n)).cuda()
    za = torch.from_numpy(np.arccos(rng.uniform(0.05, 1.0, n))).cuda()
    lat = torch.tensor([-0.4660608448386394], dtype=torch.float64, device="cuda")
    out = torch.empty((nu, nuf, n, 8), dtype=torch.float64, device="cuda")  # > L2 at the full size
    stream = torch.cuda.current_stream()
    st = ctypes.c_void_p(stream.cuda_stream)

    def call():
        _lib.check(lib.hdc_fee_calc_jones(beam.handle, az.data_ptr(), za.data_ptr(), n, lat.data_ptr(), 0,
                                          out.data_ptr(), st), "hdc_fee_calc_jones")

    ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
    for _ in range(3):
        call()
    times = []
    for _ in range(5):
        torch.cuda.synchronize()
        ev[0].record(stream)
        call()
        ev[1].record(stream)
        torch.cuda.synchronize()
        times.append(ev[0].elapsed_time(ev[1]) * 1e-3)
    t = statistics.median(times)
    modes = FEE_NMAX * (FEE_NMAX + 2)
    jones = nu * nuf * n
    flop = jones * modes * FEE_FLOP_PER_MODE
    g = ctypes.c_double()
    _lib.check(lib.hdc_probe_fp64_gflops(ctypes.byref(g)), "hdc_probe_fp64_gflops")
    res = {"workload": FEE_WORKLOAD, "unique_tiles": nu, "unique_freqs": nuf,
           "directions": n, "s_per_call": t, "jones_per_s": jones / t, "jones_modes_per_s": jones * modes / t,
           "roofline": {"bound": "fp64", "kernel": "fee_jones_kernel", "achieved": flop / t / 1e12,
                        "peak": g.value / 1e3, "unit": "TFLOP/s", "frac": flop / t / 1e9 / g.value,
                        "peak_source": "FP64 FMA probe kernel measured in this run",
                        "flop_per_launch": flop,
                        "flop_rule": f"{FEE_FLOP_PER_MODE} FLOP per mode per direction per (unique tile, "
                                     "unique frequency); the Legendre recurrences are not counted"}}
    # the predict of one timestep of the mixed configuration with this beam per
    # tile (chosen form: tensor block form for the points, the per-tile kernel
    # of the chosen form for Gaussians and shapelets) beside the shared
    # analytic beam, per kernel class (the modeller's CUDA events)
    if n == 4600:
        from mwa_hyperdrive_b200.model import SkyModeller

        obs, sky = workload()
        if obs.num_tiles == ntiles and np.allclose(obs.freqs, chans):
            vis = torch.zeros((obs.freqs.size, obs.num_baselines, 8), dtype=torch.float32, device="cuda")
            per = {}
            for name, bm in (("fee_per_tile", "fee"), ("analytic_shared", "analytic")):
                m = SkyModeller(sky, obs.tile_xyzs, obs.freqs, obs.phase_centre, obs.latitude, form="tensor", beam=bm,
                                fee_beam=beam if bm == "fee" else None)
                m.model_timestep_with(obs.lsts[0], vis, return_uvws=False)
                lib.hdc_modeller_set_profiling(m._h, 1)
                prof = (ctypes.c_double * 4)()
                runs = []
                for _ in range(3):
                    lib.hdc_modeller_profile(m._h, prof, 1)
                    m.model_timestep_with(obs.lsts[0], vis, return_uvws=False)
                    torch.cuda.synchronize()
                    lib.hdc_modeller_profile(m._h, prof, 1)
                    runs.append(list(prof))
                med = [statistics.median(r[i] for r in runs) for i in range(4)]
                per[name] = {"ms_per_timestep": sum(med), "points": med[0], "gaussians": med[1],
                             "shapelets": med[2], "geometry_and_beam": med[3]}
                m.close()
            res["predict_one_timestep"] = per
            del vis
    if not args.no_cpu_baseline:
        from oracle import fee_ref as fr

        k = 2  # sets in the sample
        azh, zah = az.cpu().numpy(), za.cpu().numpy()
        t0 = time.perf_counter()
        for i in range(k):
            fr.calc_jones(coeffs, azh, zah, chans[i * 100], delays[i], amps[i], norm_to_zenith=True,
                          latitude=-0.4660608448386394)
        dt = time.perf_counter() - t0
        res["cpu_baseline"] = {"value": dt * (nu * nuf) / k, "unit": "s per call", "cores": 1, "kind": "port",
                               "sample": f"{k} of {nu * nuf} (tile, frequency) sets x {n} directions "
                                         f"(numpy restatement, {dt:.1f} s), scaled"}
        res["speedup_vs_cpu"] = res["cpu_baseline"]["value"] / t
    beam.close()
    return res


def guarded(fn, args):
    """Run an optional bench section; a failure is reported in the line."""
    try:
        return fn(args)
    except Exception as e:  # reported, not hidden: the key holds the error
        return {"error": f"{type(e).__name__}: {e}"}


# DRAM bytes (dram__bytes_read.sum + dram__bytes_write.sum) per launch of each
# kernel class on this workload (one timestep, 384 channels), from the ncu
# launch list of the bench command itself (one pass: gpu__time_duration and
# the two DRAM counters).  The visibilities alone are 100 MB read + 100 MB
# written per launch.
# The tensor point predict of one timestep runs in chunks of channels; the
# figure is its Gram kernels' DRAM over the timestep: they read the table of
# A planes and phasors (written by phasor_table_kernel, 2.42 GB per
# timestep) once from DRAM.
NCU_TRAFFIC_SOURCE = "ncu launch list of this bench command (launch-list summary of the predict kernels)"
NCU_DRAM_BYTES_PER_LAUNCH = {
    ("points", "tensor"): 2927e6, ("gaussians", "tensor"): 156.0e6, ("shapelets", "tensor"): 164.5e6,
    ("points", "direct"): 268.0e6, ("gaussians", "direct"): 152.0e6, ("shapelets", "direct"): 142.0e6,
}


# ------------------------------------------------------------ GPU arm
def gpu_arm(args, rank, world, local_rank):
    import torch

    from mwa_hyperdrive_b200 import _lib
    from mwa_hyperdrive_b200.model import SkyModeller

    torch.cuda.set_device(local_rank)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local_rank))
    L = _lib.lib()
    obs, sky = workload()
    form = args.form
    if form == "auto":
        form = "direct"
        try:
            SkyModeller(sky.select(sky.comp_type == 0), obs.tile_xyzs, obs.freqs[:1], obs.phase_centre, obs.latitude,
                        form="tensor").close()
            form = "tensor"
        except _lib.HdcError:
            form = "direct"
    stream = torch.cuda.current_stream()
    nf, nbl, nt = obs.freqs.size, obs.num_baselines, obs.lsts.size

    def make(fm):
        m = SkyModeller(sky, obs.tile_xyzs, obs.freqs, obs.phase_centre, obs.latitude, beam="analytic", form=fm)
        return m

    vis = torch.zeros((nt, nf, nbl, 8), dtype=torch.float32, device="cuda")
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")

    def step(m):
        vis.zero_()
        for t in range(nt):
            m.model_timestep_with(float(obs.lsts[t]), vis[t], stream=stream, return_uvws=False)

    def timed(m, steps, warmup):
        for _ in range(warmup):
            step(m)
        torch.cuda.synchronize()
        # discard event timings recorded during warm-up
        discard = (ctypes.c_double * 4)()
        L.hdc_modeller_profile(m._h, discard, 1)
        if dist:
            dist.barrier()
        torch.cuda.synchronize()
        evs = []
        launches0 = L.hdc_kernel_launches()
        for k in range(steps):
            flush.fill_(float(k))
            a = torch.cuda.Event(enable_timing=True)
            b = torch.cuda.Event(enable_timing=True)
            a.record(stream)
            step(m)
            b.record(stream)
            evs.append((a, b))
        torch.cuda.synchronize()
        launches = L.hdc_kernel_launches() - launches0
        ms = [a.elapsed_time(b) for a, b in evs]
        total = max_over_ranks(sum(ms), dist)
        if dist:
            dist.barrier()
        return total / steps, launches // steps

    results = {}
    plain = make("direct")
    clocks = ClockSampler(local_rank)
    ms_plain, launches_plain = timed(plain, args.steps, args.warmup)
    results["direct"] = ms_plain
    chosen = plain
    if form == "tensor":
        chosen = make("tensor")
    L.hdc_modeller_set_profiling(chosen._h, 1)
    clocks.start()
    ms_chosen, launches = timed(chosen, args.steps, args.warmup)
    clk = clocks.stop()
    prof = (ctypes.c_double * 4)()
    L.hdc_modeller_profile(chosen._h, prof, 1)
    L.hdc_modeller_set_profiling(chosen._h, 0)

    work = vis_comp_per_step(obs, sky)
    value = aggregate(work, world, ms_chosen * 1e-3)

    # e2e: trait-style host-buffer calls (pinned host memory)
    e2e_s = None
    if not args.skip_e2e:
        hvis = torch.zeros((nt, nf, nbl, 8), dtype=torch.float32).pin_memory()
        hnp = hvis.numpy()
        for _ in range(max(1, args.warmup)):
            for t in range(nt):
                chosen.model_timestep_with_host(float(obs.lsts[t]), hnp[t], stream=stream)
        torch.cuda.synchronize()
        if dist:
            dist.barrier()
        t0 = time.perf_counter()
        e2e_steps = max(2, args.steps)
        # the predict accumulates into the host buffer (the trait's
        # model_timestep_with semantics), so no host-side clearing is timed
        for _ in range(e2e_steps):
            for t in range(nt):
                chosen.model_timestep_with_host(float(obs.lsts[t]), hnp[t], stream=stream)
        e2e_s = max_over_ranks((time.perf_counter() - t0) / e2e_steps, dist)
    bytes_vis = nt * nf * nbl * 32

    # roofline of every kernel class of the chosen form; `roofline` is the
    # dominant one (largest share of the step)
    names = ["points", "gaussians", "shapelets", "prep"]
    per_step_ms = [prof[k] / args.steps for k in range(4)]
    dom = int(np.argmax(per_step_ms[:3]))
    npts = int(np.sum(sky.comp_type == 0))
    nga = int(np.sum(sky.comp_type == 1))
    nsh = int(np.sum(sky.comp_type == 2))
    ncoef = int(np.sum(sky.coeff_count))
    launches_per_step = nt
    g64, g32 = ctypes.c_double(), ctypes.c_double()
    _lib.check(L.hdc_probe_fp64_gflops(ctypes.byref(g64)), "fp64 probe")
    _lib.check(L.hdc_probe_fp32_gflops(ctypes.byref(g32)), "fp32 probe")
    peaks = json.loads((ROOT / "MEASURED_PEAKS.json").read_text()) if (ROOT / "MEASURED_PEAKS.json").exists() else {}
    by_class = {}
    for k, ncomp in enumerate([npts, nga, nsh]):
        if ncomp == 0 or per_step_ms[k] <= 0.0:
            continue
        t_launch = per_step_ms[k] / launches_per_step * 1e-3
        if k == 0 and form == "tensor":
            # useful complex-GEMM flops: 3 products (XX, XY, YY) of 8 x 128 x 128 x Nc per (t, f)
            flops = 3 * 8 * obs.num_tiles * obs.num_tiles * npts * nf
            entry = {"bound": "tensor", "kernel": "gram_i8_kernel (points, tcgen05 kind::i8)",
                     "peak": peaks.get("bf16_tflops", 1590.0),
                     "peak_source": "MEASURED_PEAKS.json bf16 burst" if peaks else "fallback 1590 TFLOP/s"}
        else:
            # algorithmic FLOPs per visibility-component: phase 5 + Jones x phasor 24 + accumulate 8;
            # Gaussians +10 (envelope); shapelets +12 per coefficient
            fl_per = {0: 37.0, 1: 47.0, 2: 37.0 + 12.0 * ncoef / max(nsh, 1)}[k]
            flops = fl_per * nbl * nf * ncomp
            fast = form == "tensor"
            entry = {"bound": "fp32" if fast else "fp64",
                     "kernel": f"fast_kernel ({names[k]}, FP32 form)" if fast else f"direct_kernel ({names[k]}, FP64)",
                     "peak": (g32.value if fast else g64.value) / 1e3,
                     "peak_source": f"{'FP32' if fast else 'FP64'} FMA probe kernel measured in this run"}
        traffic = NCU_DRAM_BYTES_PER_LAUNCH.get((names[k], form))
        entry.update({"achieved": flops / t_launch / 1e12, "unit": "TFLOP/s", "traffic": traffic,
                      "traffic_source": NCU_TRAFFIC_SOURCE if traffic else None, "ms_per_step": per_step_ms[k]})
        if k == 0 and form == "tensor":
            # what the tensor pipe executes: 18 kind::i8 MMAs of 128 x 128 x 32 per 32-component stage of each
            # (channel, polarisation, column block) CTA, against 8190 int8 MAC/clk/SM (a probe of back-to-back
            # kind::i8 MMAs) at this run's median SM clock
            macs = nf * 6 * ((npts + 31) // 32) * 18 * 128 * 128 * 32
            n_sm = torch.cuda.get_device_properties(0).multi_processor_count
            mhz = (clk or {}).get("sm_mhz") or 1965.0
            entry["int8_mma"] = {"executed_macs_per_s": macs / t_launch,
                                 "peak_macs_per_s": 8190.0 * n_sm * mhz * 1e6,
                                 "frac": macs / t_launch / (8190.0 * n_sm * mhz * 1e6)}
        entry["frac"] = entry["achieved"] / entry["peak"]
        by_class[names[k]] = entry
    roofline = dict(by_class[names[dom]])
    roofline["per_step_ms_by_class"] = dict(zip(names, per_step_ms))
    roofline["by_class"] = by_class

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_chosen, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64" if form == "direct" else "f64 phases, s8 digit planes with exact s32 accumulation (points); f32 terms with f64 arguments and chunk sums (Gaussians, shapelets)",
            "data": "synthetic (seeded)", "config": config_dict(obs, sky, form),
            "plain": {"form": "direct", "value": work * world / (ms_plain * 1e-3), "ms_per_step": ms_plain},
            "e2e": None if e2e_s is None else {"value": work * world / e2e_s, "unit": UNIT,
                                               "h2d_bytes_per_step": bytes_vis, "d2h_bytes_per_step": bytes_vis},
            "roofline": roofline, "gpu_launches": int(launches), "clocks": clk,
        }
        if world == 1 and not args.no_cpu_baseline:
            line["cpu_baseline"] = cpu_baseline(obs, sky, args.cpu_seconds)
            # the checker on the timed configuration: the last timed step's
            # output (still in `vis`) against the FP64 oracle
            line["error"] = sampled_error(vis, obs, sky)
            line["reference_gpu"] = guarded(lambda a: reference_gpu_leg(obs, sky), args)
            rg = line["reference_gpu"]
            if "all_types" in rg:
                # the same timestep through the native modeller: the plain
                # (all-FP64) and the chosen form, against the reference's kernels
                ref_ms = rg["all_types"]["ref_ms"]
                rg["native_plain_form"] = {"ms_per_timestep": ms_plain / nt,
                                           "speedup_vs_reference_kernels": ref_ms / (ms_plain / nt)}
                rg["native_chosen_form"] = {"ms_per_timestep": ms_chosen / nt,
                                            "speedup_vs_reference_kernels": ref_ms / (ms_chosen / nt)}
            torch.cuda.synchronize()
        # the sections of a 1-GPU run (a multi-GPU run measures the replicated
        # predict only)
        single = world == 1
        if single and not (args.skip_dical and args.skip_peel and args.skip_warmstart and args.skip_prep
                           and args.skip_fee):
            del vis, flush
            torch.cuda.empty_cache()
        if single and not args.skip_dical:
            line["dical"] = guarded(dical_arm, args)
            torch.cuda.empty_cache()
        if single and not args.skip_peel:
            line["peel"] = guarded(peel_arm, args)
            torch.cuda.empty_cache()
        if single and not args.skip_warmstart:
            line["warmstart"] = guarded(warmstart_arm, args)
            torch.cuda.empty_cache()
        if single and not args.skip_prep:
            line["prep"] = guarded(prep_arm, args)
            torch.cuda.empty_cache()
        if single and not args.skip_fee:
            line["fee"] = guarded(fee_arm, args)
        print(json.dumps(line), flush=True)
    plain.close()
    if chosen is not plain:
        chosen.close()
    if dist:
        dist.destroy_process_group()


def main():
    args = parse()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", str(args.gpus if args.gpus == 1 else 1)))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        reference_arm(args, rank)
        return
    gpu_arm(args, rank, world, local_rank)


if __name__ == "__main__":
    main()
