"""The oracle's restatement of the reference's CPU peel loop (peel_cpu,
params/peel/mod.rs:1121-1475), CPU only.

As in the reference's own peel tests (params/peel/tests.rs:1549-1816), a
residual is made from sources whose visibilities carry known ionospheric
offsets (alpha, beta) scaled by lambda^2 and gains; the residual is the data
minus the sources' models without ionosphere.  Peeling must recover every
source's (alpha, beta, gain) and remove it from the residual.  The
reference's tolerances there are 1e-10 rad and 1e-8 on noiseless data; the
FP32 visibilities here give ~1e-7 of the gain.  A source with no ionosphere
and a unit gain must leave the residual unchanged to rounding.
"""

import math

import numpy as np

from mwa_hyperdrive_b200 import srclist as sl
from mwa_hyperdrive_b200 import synth
from oracle import oracle as O

VEL_C = 299792458.0


def problem(nsrc, inject, seed=4, ntiles=24, nt=2, nf=16):
    rng = np.random.default_rng(seed)
    pc = (0.1, math.radians(-27.0))
    xyzs = synth.tiles_in_disk(ntiles, 1500.0, seed)
    freqs = 165e6 + np.arange(nf) * 1.28e6
    lmsts = pc[0] + np.arange(nt) * 8.0 * synth.SIDEREAL_RATE
    lam = VEL_C / freqs
    sources, positions, truths = [], [], []
    for _ in range(nsrc):
        ra = pc[0] + math.radians(rng.uniform(-3, 3))
        dec = pc[1] + math.radians(rng.uniform(-3, 3))
        sources.append(sl.SkyModelArrays.from_components(
            [sl.SourceComponent(ra, dec, sl.Point(), sl.PowerLaw(-0.8, sl.FluxDensity(150e6, float(rng.uniform(2, 6)))))]))
        positions.append((ra, dec))
        truths.append((rng.normal(0, 2e-5), rng.normal(0, 2e-5), rng.uniform(0.95, 1.05)) if inject else (0, 0, 1))
    nbl = ntiles * (ntiles - 1) // 2
    resid = np.zeros((nt, nf, nbl, 8))
    for sky, pos, (a, b, g) in zip(sources, positions, truths):
        for t in range(nt):
            m, _ = O.model_timestep(sky, xyzs, freqs, pc, lmsts[t], synth.MWA_LAT_RAD, out_f64=True)
            uvw = O.xyzs_to_cross_uvws(xyzs, lmsts[t] - pos[0], pos[1])
            ph = g * np.exp(-2j * np.pi * (uvw[:, 0] * a + uvw[:, 1] * b)[None, :] * lam[:, None]) - 1.0
            v = (m[..., 0::2] + 1j * m[..., 1::2]) * ph[..., None]
            resid[t, ..., 0::2] += v.real
            resid[t, ..., 1::2] += v.imag
    return (resid.astype(np.float32), np.ones((nt, nf, nbl), np.float32), freqs, xyzs, lmsts, pc, sources, positions,
            truths)


def test_peel_cpu_recovers_injected_ionosphere():
    resid, w, freqs, xyzs, lmsts, pc, sources, positions, truths = problem(3, True)
    out, consts = O.peel_cpu(resid, w, freqs, xyzs, lmsts, float(np.median(lmsts)), pc, sources, positions,
                             [(0.0, 0.0, 1.0)] * 3, num_passes=3, num_loops=10, convergence=1.0, favg=4,
                             lat=synth.MWA_LAT_RAD)
    for (a, b, g), (ta, tb, tg) in zip(consts, truths):
        assert abs(a - ta) < 1e-8 and abs(b - tb) < 1e-8, (a, ta, b, tb)
        assert abs(g - tg) < 1e-5, (g, tg)
    assert np.linalg.norm(out) < 1e-3 * np.linalg.norm(resid)


def test_peel_cpu_without_ionosphere_leaves_the_residual():
    resid, w, freqs, xyzs, lmsts, pc, sources, positions, truths = problem(1, False, seed=6)
    resid = resid + np.random.default_rng(1).normal(0.0, 0.1, resid.shape).astype(np.float32)
    out, consts = O.peel_cpu(resid, w, freqs, xyzs, lmsts, float(np.median(lmsts)), pc, sources, positions,
                             [(0.0, 0.0, 1.0)], num_passes=1, num_loops=10, convergence=1.0, favg=4,
                             lat=synth.MWA_LAT_RAD)
    a, b, g = consts[0]
    assert abs(a) < 1e-6 and abs(b) < 1e-6 and abs(g - 1.0) < 1e-2
