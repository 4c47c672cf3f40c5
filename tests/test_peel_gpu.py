"""Peeling on the GPU: the drop-in peel kernels (gpu/peel.h) against the
oracle's restatement of the reference kernels, the native peel loop against
the same loop composed from oracle pieces, and recovery of injected
ionospheric offsets (the structure of params/peel/tests.rs:1549-1816).

Visibilities are f32 as in the reference, with f64 internal arithmetic;
kernels are compared within a few f32 ulps (relative 1e-6), fitted constants
within 1e-6 relative."""

import ctypes
import math

import numpy as np
import pytest

from mwa_hyperdrive_b200 import srclist as sl
from mwa_hyperdrive_b200 import synth

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("no CUDA device", allow_module_level=True)

from mwa_hyperdrive_b200 import _lib  # noqa: E402
from mwa_hyperdrive_b200 import peel as P  # noqa: E402

VEL_C = 299792458.0


_KEEP = []


def dev(x, dt=np.float64):
    """Device copy that stays alive for the test (kernels run asynchronously,
    so a temporary freed right after .data_ptr() could be reused before the
    kernel reads it)."""
    t = torch.from_numpy(np.ascontiguousarray(x, dt)).cuda()
    _KEEP.append(t)
    return t


@pytest.fixture(autouse=True)
def _release_kept():
    yield
    torch.cuda.synchronize()
    _KEEP.clear()


def rel(a, b):
    return np.linalg.norm(np.asarray(a, np.float64) - np.asarray(b, np.float64)) / np.linalg.norm(np.asarray(b, np.float64))


def setup(ntiles=16, nt=2, nf=8, seed=0):
    rng = np.random.default_rng(seed)
    pc = (0.1, math.radians(-27.0))
    xyzs = synth.tiles_in_disk(ntiles, 1500.0, seed + 1)
    freqs = 165e6 + np.arange(nf) * 1.28e6
    lmsts = pc[0] + np.arange(nt) * 8.0 * synth.SIDEREAL_RATE
    return rng, pc, xyzs, freqs, lmsts


def test_xyzs_to_uvws_and_rotate(oracle):
    rng, pc, xyzs, freqs, lmsts = setup()
    nt, ntiles = lmsts.size, xyzs.shape[0]
    nbl = ntiles * (ntiles - 1) // 2
    xyz_t = np.broadcast_to(xyzs, (nt, ntiles, 3)).copy()
    L = _lib.lib()
    d_xyz, d_lmst = dev(xyz_t), dev(lmsts)
    d_uvw = torch.zeros((nt, nbl, 3), dtype=torch.float64, device="cuda")
    src = (0.13, math.radians(-25.0))
    _lib.check_str(L.xyzs_to_uvws(d_xyz.data_ptr(), d_lmst.data_ptr(), d_uvw.data_ptr(), _lib.RADec(*src), ntiles, nbl,
                                  nt), "xyzs_to_uvws")
    ref = oracle.xyzs_to_uvws(xyz_t, lmsts, src)
    np.testing.assert_allclose(d_uvw.cpu().numpy(), ref, rtol=0, atol=1e-10)
    frm = oracle.xyzs_to_uvws(xyz_t, lmsts, pc)
    vis = (rng.normal(size=(nt, freqs.size, nbl, 8))).astype(np.float32)
    lam = VEL_C / freqs
    d_vis = dev(vis, np.float32)
    _lib.check_str(L.rotate(d_vis.data_ptr(), nt, nbl, freqs.size, dev(frm).data_ptr(), d_uvw.data_ptr(),
                            dev(lam).data_ptr()), "rotate")
    torch.cuda.synchronize()
    assert rel(d_vis.cpu().numpy(), oracle.rotate(vis, frm, ref, lam)) < 1e-6


def test_average_add_model_subtract(oracle):
    rng, pc, xyzs, freqs, lmsts = setup()
    nt, nf, ntiles = lmsts.size, freqs.size, xyzs.shape[0]
    nbl = ntiles * (ntiles - 1) // 2
    L = _lib.lib()
    hi = rng.normal(size=(nt, nf, nbl, 8)).astype(np.float32)
    w = rng.uniform(0.0, 2.0, (nt, nf, nbl)).astype(np.float32)
    w[:, :, ::7] = 0.0
    lo = torch.zeros((nf // 4, nbl, 8), dtype=torch.float32, device="cuda")
    _lib.check_str(L.average(dev(hi, np.float32).data_ptr(), dev(w, np.float32).data_ptr(), lo.data_ptr(), nt, nbl,
                             nf, 4), "average")
    torch.cuda.synchronize()
    assert rel(lo.cpu().numpy(), oracle.average(hi, w, 4)) < 1e-6
    uvws = rng.normal(size=(nt, nbl, 3)) * 300.0
    lam = VEL_C / freqs
    model = rng.normal(size=(nt, nf, nbl, 8)).astype(np.float32)
    c = (1.3e-5, -2.1e-5, 1.04)
    old = (0.4e-5, 0.9e-5, 0.97)
    for consts in [c, (0.0, 0.0, 1.1)]:
        r = dev(hi, np.float32)
        _lib.check_str(L.add_model(r.data_ptr(), dev(model, np.float32).data_ptr(), _lib.IonoConsts(*consts),
                                   dev(lam).data_ptr(), dev(uvws).data_ptr(), nt, nf, nbl), "add_model")
        torch.cuda.synchronize()
        assert rel(r.cpu().numpy(), oracle.add_model(hi, model, consts, lam, uvws)) < 1e-6
    r = dev(hi, np.float32)
    _lib.check_str(L.subtract_iono(r.data_ptr(), dev(model, np.float32).data_ptr(), _lib.IonoConsts(*c),
                                   _lib.IonoConsts(*old), dev(uvws).data_ptr(), dev(lam).data_ptr(), nt, nbl, nf),
                   "subtract_iono")
    torch.cuda.synchronize()
    assert rel(r.cpu().numpy(), oracle.subtract_iono(hi, model, c, old, uvws, lam)) < 1e-6


def iono_rotate(vis_fb, uvw_b, consts, lam):
    a, b, g = consts
    arg = -2 * np.pi * (uvw_b[:, 0] * a + uvw_b[:, 1] * b)
    ph = np.exp(1j * arg[None, :] * lam[:, None]) * g
    v = vis_fb[..., 0::2] + 1j * vis_fb[..., 1::2]
    v = v * ph[..., None]
    out = np.empty_like(vis_fb)
    out[..., 0::2] = v.real
    out[..., 1::2] = v.imag
    return out.astype(np.float32)


def test_iono_loop_matches_oracle(oracle):
    rng, pc, xyzs, freqs, lmsts = setup(ntiles=24, nf=12)
    ntiles = xyzs.shape[0]
    nbl = ntiles * (ntiles - 1) // 2
    lam = VEL_C / freqs
    uvw = oracle.xyzs_to_cross_uvws(xyzs, 0.1, -0.4)
    model = np.zeros((freqs.size, nbl, 8), np.float32)
    amp = rng.lognormal(0, 0.3, (freqs.size, nbl))
    model[..., 0] = amp
    model[..., 6] = amp
    true = (2e-5, -1.5e-5, 1.05)
    resid = iono_rotate(model, uvw, true, lam)
    w = np.ones((freqs.size, nbl), np.float32)
    L = _lib.lib()
    c = _lib.IonoConsts(0.0, 0.0, 1.0)
    rot = torch.zeros_like(dev(model, np.float32))
    fits = torch.zeros((freqs.size, nbl, 8), dtype=torch.float64, device="cuda")
    _lib.check_str(L.iono_loop(dev(resid, np.float32).data_ptr(), dev(w, np.float32).data_ptr(),
                               dev(model, np.float32).data_ptr(), rot.data_ptr(), fits.data_ptr(), ctypes.byref(c),
                               nbl, freqs.size, 10, dev(uvw).data_ptr(), dev(lam).data_ptr(), 1.0), "iono_loop")
    (ra, rb, rg), rrot = oracle.iono_loop(resid, w, model, (0.0, 0.0, 1.0), 10, uvw, lam, 1.0)
    assert abs(c.alpha - ra) <= 1e-6 * abs(ra) and abs(c.beta - rb) <= 1e-6 * abs(rb) and abs(c.gain - rg) < 1e-9
    # and the fit recovers the injected constants
    assert abs(c.alpha - true[0]) < 1e-3 * abs(true[0]) and abs(c.beta - true[1]) < 1e-3 * abs(true[1])
    assert abs(c.gain - true[2]) < 1e-5


# ---------------------------------------------------------------- peel loop
def make_peel_problem(seed=3, ntiles=20, nt=2, nf=8, nsrc=3, inject=True, points=False):
    rng, pc, xyzs, freqs, lmsts = setup(ntiles, nt, nf, seed)
    nbl = ntiles * (ntiles - 1) // 2
    lam = VEL_C / freqs
    sources, positions, truths = [], [], []
    for s in range(nsrc):
        ra = pc[0] + math.radians(rng.uniform(-3, 3))
        dec = pc[1] + math.radians(rng.uniform(-3, 3))
        comps = [sl.SourceComponent(ra + math.radians(0.02 * k), dec, sl.Point(),
                                    sl.PowerLaw(-0.8, sl.FluxDensity(150e6, float(rng.uniform(2, 6)))))
                 for k in range(1 if points else 2)]
        sources.append(sl.SkyModelArrays.from_components(comps))
        positions.append((ra, dec))
        truths.append((rng.normal(0, 2e-5), rng.normal(0, 2e-5), rng.uniform(0.95, 1.05)) if inject else (0, 0, 1))
    return rng, pc, xyzs, freqs, lmsts, lam, nbl, sources, positions, truths


def simulate_residual(oracle, pc, xyzs, freqs, lmsts, lam, sources, positions, truths, beam_for=None):
    """data = sum_s model_s * iono_s (uv at the source position); residual =
    data - sum_s model_s, everything at the observation phase centre;
    beam_for(sky, lst) gives the oracle's per-tile beam tables (or none)."""
    nt, nf = lmsts.size, freqs.size
    n = xyzs.shape[0]
    nbl = n * (n - 1) // 2
    resid = np.zeros((nt, nf, nbl, 8), np.float64)
    for sky, pos, tr in zip(sources, positions, truths):
        for t in range(nt):
            m, _ = oracle.model_timestep(sky, xyzs, freqs, pc, lmsts[t], synth.MWA_LAT_RAD, out_f64=True,
                                         beam=beam_for(sky, lmsts[t]) if beam_for else None)
            uvw_src = oracle.xyzs_to_cross_uvws(xyzs, lmsts[t] - pos[0], pos[1])
            resid[t] += iono_rotate(m, uvw_src, tr, lam).astype(np.float64) - m
    return resid.astype(np.float32)


def oracle_peel(oracle, resid, weights, pc, xyzs, freqs, lmsts, avg_lmst, sources, positions, consts, num_passes,
                num_loops, conv, favg, beam_for=None):
    """The native loop's sequence (peel_gpu, params/peel/gpu.rs:355-757)
    composed from the oracle's kernels (beam_for(sky, lst): the sources'
    per-tile beam tables, or none)."""
    resid = resid.copy()
    nt, nf, nbl = resid.shape[:3]
    n = xyzs.shape[0]
    lam = VEL_C / freqs
    flo = freqs.reshape(-1, favg).mean(axis=1)
    lam_lo = VEL_C / flo
    xyz_t = np.broadcast_to(xyzs, (nt, n, 3)).copy()
    w_lo = np.maximum(weights.astype(np.float64).reshape(nt, nf // favg, favg, nbl).sum(axis=(0, 2)), 0).astype(
        np.float32)
    consts = [tuple(c) for c in consts]
    for _ in range(num_passes):
        frm = oracle.xyzs_to_uvws(xyz_t, lmsts, pc)
        for i, (sky, pos) in enumerate(zip(sources, positions)):
            old = consts[i]
            to = oracle.xyzs_to_uvws(xyz_t, lmsts, pos)
            resid = oracle.rotate(resid, frm, to, lam)
            model = np.zeros((nt, nf, nbl, 8), np.float32)
            for t in range(nt):
                for ty in range(3):
                    if np.any(np.asarray(sky.comp_type) == ty):
                        oracle.model_type(ty, sky, xyzs, freqs, pos, lmsts[t], synth.MWA_LAT_RAD, to[t],
                                          vis=model[t], beam=beam_for(sky, lmsts[t]) if beam_for else None)
            rsrc = oracle.add_model(resid, model, old, lam, to)
            mrot = oracle.add_model(np.zeros_like(model), model, old, lam, to)
            rlo = oracle.average(rsrc, weights, favg)
            mlo = oracle.average(mrot, weights, favg)
            uv_lo = oracle.xyzs_to_uvws(xyzs[None], np.array([avg_lmst]), pos)[0]
            (da, db, dg), _ = oracle.iono_loop(rlo, w_lo, mlo, (0.0, 0.0, 1.0), num_loops, uv_lo, lam_lo, conv)
            c = (old[0] + da, old[1] + db, old[2] * dg)
            if abs(c[0]) > 1e-3 or abs(c[1]) > 1e-3 or c[2] < 0 or c[2] > 1.5:
                c = old
            consts[i] = c
            resid = oracle.subtract_iono(resid, model, c, old, to, lam)
            frm = to
        back = oracle.xyzs_to_uvws(xyz_t, lmsts, pc)
        resid = oracle.rotate(resid, frm, back, lam)
    return resid, consts


def test_native_peel_matches_oracle_loop(oracle):
    rng, pc, xyzs, freqs, lmsts, lam, nbl, sources, positions, truths = make_peel_problem()
    resid = simulate_residual(oracle, pc, xyzs, freqs, lmsts, lam, sources, positions, truths)
    weights = np.ones(resid.shape[:3], np.float32)
    avg_lmst = float(np.median(lmsts))
    start = [P.IonoConsts() for _ in sources]
    d_resid = dev(resid, np.float32)
    got = P.peel_timeblock(d_resid, dev(weights, np.float32), freqs, xyzs, lmsts, avg_lmst, pc, sources, positions,
                           start, num_passes=2, num_loops=5, convergence=1.0, freq_average_factor=4,
                           array_latitude_rad=synth.MWA_LAT_RAD)
    ref_resid, ref_consts = oracle_peel(oracle, resid, weights, pc, xyzs, freqs, lmsts, avg_lmst, sources, positions,
                                        [(0.0, 0.0, 1.0)] * len(sources), 2, 5, 1.0, 4)
    for g, r in zip(got, ref_consts):
        assert abs(g.alpha - r[0]) <= 1e-5 * abs(r[0]) + 1e-12
        assert abs(g.beta - r[1]) <= 1e-5 * abs(r[1]) + 1e-12
        assert abs(g.gain - r[2]) <= 1e-6
    assert rel(d_resid.cpu().numpy(), ref_resid) < 1e-4


def test_native_peel_recovers_injected_iono(oracle):
    rng, pc, xyzs, freqs, lmsts, lam, nbl, sources, positions, truths = make_peel_problem(seed=7, ntiles=32, nf=16,
                                                                                           nsrc=2)
    resid = simulate_residual(oracle, pc, xyzs, freqs, lmsts, lam, sources, positions, truths)
    before = np.linalg.norm(resid)
    weights = np.ones(resid.shape[:3], np.float32)
    d_resid = dev(resid, np.float32)
    got = P.peel_timeblock(d_resid, dev(weights, np.float32), freqs, xyzs, lmsts, float(np.median(lmsts)), pc,
                           sources, positions, [P.IonoConsts() for _ in sources], num_passes=3, num_loops=10,
                           convergence=1.0, freq_average_factor=4, array_latitude_rad=synth.MWA_LAT_RAD)
    after = np.linalg.norm(d_resid.cpu().numpy())
    for g, tr in zip(got, truths):
        assert abs(g.alpha - tr[0]) < 0.02 * abs(tr[0]) + 2e-7, (g, tr)
        assert abs(g.beta - tr[1]) < 0.02 * abs(tr[1]) + 2e-7, (g, tr)
        assert abs(g.gain - tr[2]) < 5e-3, (g, tr)
    assert after < 0.05 * before, (after, before)


# ------------------------------------------------------------ batched peel
@pytest.mark.parametrize("points", [False, True])
def test_batched_peel_single_source_equals_sequential(oracle, points):
    """With one source the batched (Jacobi) pass is the reference's sequence:
    same constants and residual up to rounding (FP64 instead of f32
    intermediates).  points: one point at the source position (the
    per-(timestep, channel) model table) instead of a two-component source
    (materialised model)."""
    rng, pc, xyzs, freqs, lmsts, lam, nbl, sources, positions, truths = make_peel_problem(seed=5, nsrc=1,
                                                                                           points=points)
    resid = simulate_residual(oracle, pc, xyzs, freqs, lmsts, lam, sources, positions, truths)
    weights = np.ones(resid.shape[:3], np.float32)
    weights[:, :, ::5] = 0.5
    avg_lmst = float(np.median(lmsts))
    out = {}
    for batched in (False, True):
        d_resid = dev(resid, np.float32)
        c = P.peel_timeblock(d_resid, dev(weights, np.float32), freqs, xyzs, lmsts, avg_lmst, pc, sources, positions,
                             [P.IonoConsts()], num_passes=2, num_loops=5, convergence=1.0, freq_average_factor=4,
                             array_latitude_rad=synth.MWA_LAT_RAD, batched=batched)
        out[batched] = (c[0], d_resid.cpu().numpy())
    (cs, rs), (cb, rb) = out[False], out[True]
    assert abs(cb.alpha - cs.alpha) <= 1e-5 * abs(cs.alpha) + 1e-12, (cb, cs)
    assert abs(cb.beta - cs.beta) <= 1e-5 * abs(cs.beta) + 1e-12, (cb, cs)
    assert abs(cb.gain - cs.gain) <= 1e-6, (cb, cs)
    # the peeled residuals are at rounding level; compare on the input's scale
    assert np.linalg.norm(rb.astype(np.float64) - rs) / np.linalg.norm(resid) < 1e-4
    bx, sy, ms = P.batched_tuning()
    # a (bins x sources) CTA of 256 threads, or the staged variant (bins 16, sources 0)
    assert (bx * sy == 256 or (bx, sy) == (16, 0)) and ms > 0


def test_batched_peel_recovers_injected_iono(oracle):
    rng, pc, xyzs, freqs, lmsts, lam, nbl, sources, positions, truths = make_peel_problem(seed=7, ntiles=32, nf=16,
                                                                                           nsrc=4)
    resid = simulate_residual(oracle, pc, xyzs, freqs, lmsts, lam, sources, positions, truths)
    before = np.linalg.norm(resid)
    weights = np.ones(resid.shape[:3], np.float32)
    got = {}
    for batched in (False, True):
        d_resid = dev(resid, np.float32)
        got[batched] = P.peel_timeblock(d_resid, dev(weights, np.float32), freqs, xyzs, lmsts,
                                        float(np.median(lmsts)), pc, sources, positions,
                                        [P.IonoConsts() for _ in sources], num_passes=3, num_loops=10,
                                        convergence=1.0, freq_average_factor=4,
                                        array_latitude_rad=synth.MWA_LAT_RAD, batched=batched)
        if batched:
            after = np.linalg.norm(d_resid.cpu().numpy())
    for g, s_, tr in zip(got[True], got[False], truths):
        assert abs(g.alpha - tr[0]) < 0.02 * abs(tr[0]) + 2e-7, (g, tr)
        assert abs(g.beta - tr[1]) < 0.02 * abs(tr[1]) + 2e-7, (g, tr)
        assert abs(g.gain - tr[2]) < 5e-3, (g, tr)
        # Jacobi and Gauss-Seidel agree once the passes have converged
        assert abs(g.alpha - s_.alpha) < 0.01 * abs(s_.alpha) + 1e-7, (g, s_)
    assert after < 0.05 * before, (after, before)


def test_batched_peel_in_sub_batches_of_one_is_the_sequential_order(oracle):
    """Sub-batches of one source each run the reference's Gauss-Seidel order
    (each source fitted against the residual its predecessors left): several
    sources then give the sequential loop's constants up to rounding."""
    rng, pc, xyzs, freqs, lmsts, lam, nbl, sources, positions, truths = make_peel_problem(seed=9, ntiles=24, nf=8,
                                                                                           nsrc=3, points=True)
    resid = simulate_residual(oracle, pc, xyzs, freqs, lmsts, lam, sources, positions, truths)
    weights = np.ones(resid.shape[:3], np.float32)
    avg_lmst = float(np.median(lmsts))
    out = {}
    for batched, bs in ((False, 0), (True, 1)):
        d_resid = dev(resid, np.float32)
        out[batched] = P.peel_timeblock(d_resid, dev(weights, np.float32), freqs, xyzs, lmsts, avg_lmst, pc, sources,
                                        positions, [P.IonoConsts() for _ in sources], num_passes=2, num_loops=5,
                                        convergence=1.0, freq_average_factor=4, array_latitude_rad=synth.MWA_LAT_RAD,
                                        batched=batched, batch_size=bs)
    for cb, cs in zip(out[True], out[False]):
        assert abs(cb.alpha - cs.alpha) <= 1e-5 * abs(cs.alpha) + 1e-12, (cb, cs)
        assert abs(cb.beta - cs.beta) <= 1e-5 * abs(cs.beta) + 1e-12, (cb, cs)
        assert abs(cb.gain - cs.gain) <= 1e-6, (cb, cs)


def test_batched_peel_sub_batches_recover_injected_iono(oracle):
    """Sub-batches of two of six sources: every source recovered as in the
    sequential loop."""
    rng, pc, xyzs, freqs, lmsts, lam, nbl, sources, positions, truths = make_peel_problem(seed=11, ntiles=32, nf=16,
                                                                                           nsrc=6, points=True)
    resid = simulate_residual(oracle, pc, xyzs, freqs, lmsts, lam, sources, positions, truths)
    weights = np.ones(resid.shape[:3], np.float32)
    d_resid = dev(resid, np.float32)
    got = P.peel_timeblock(d_resid, dev(weights, np.float32), freqs, xyzs, lmsts, float(np.median(lmsts)), pc,
                           sources, positions, [P.IonoConsts() for _ in sources], num_passes=3, num_loops=10,
                           convergence=1.0, freq_average_factor=4, array_latitude_rad=synth.MWA_LAT_RAD,
                           batched=True, batch_size=2)
    for g, tr in zip(got, truths):
        assert abs(g.alpha - tr[0]) < 0.02 * abs(tr[0]) + 2e-7, (g, tr)
        assert abs(g.gain - tr[2]) < 5e-3, (g, tr)
    assert np.linalg.norm(d_resid.cpu().numpy()) < 0.05 * np.linalg.norm(resid)


# ------------------------------------------------------------ the FEE beam
def fee_peel_beam(oracle, xyzs, freqs, seed=4):
    """An FEE beam per tile (synthetic coefficients at the channels, two tiles
    with a dead dipole) and beam_for(sky, lst): the oracle's FEE tables of a
    source's components in the library's unique order."""
    from mwa_hyperdrive_b200.fee import FeeBeam
    from oracle import fee_ref as fr

    n = xyzs.shape[0]
    file = synth.fee_coeffs(np.round(freqs).astype(np.uint32), 6, seed=seed)
    delays = np.tile(np.arange(16, dtype=np.uint32) % 3, (n, 1))
    delays[2, 5] = delays[7, 11] = 32
    amps = np.ones((n, 32))
    beam = FeeBeam(file, freqs, delays, amps)
    tmap, fmap = beam.maps()
    nu, nuf = int(tmap.max()) + 1, int(fmap.max()) + 1

    def beam_for(sky, lst):
        tabs = []
        for ty in range(3):
            sel = np.asarray(sky.comp_type) == ty
            if not sel.any():
                tabs.append(None)
                continue
            azel = [oracle.hadec_to_azel(lst - ra, dec, synth.MWA_LAT_RAD) for ra, dec in zip(sky.ra[sel], sky.dec[sel])]
            az = np.array([a for a, _ in azel])
            za = np.array([math.pi / 2 - e for _, e in azel])
            out = np.zeros((nu, nuf, az.size, 8))
            for u in range(nu):
                t = int(np.argmax(tmap == u))
                for uf in range(nuf):
                    f = int(np.argmax(fmap == uf))
                    out[u, uf] = fr.as_jones8(fr.calc_jones(file, az, za, freqs[f], delays[t], amps[t],
                                                            latitude=synth.MWA_LAT_RAD))
            tabs.append(out)
        return oracle.beam_struct(2, tabs, tmap, fmap, nuf)

    return beam, beam_for


def test_native_peel_with_fee_beam_matches_oracle_loop(oracle):
    """The peel loop with the FEE beam per tile (the reference's peel_gpu
    models its sources through the same beam) against the oracle's loop
    given the oracle's FEE tables."""
    rng, pc, xyzs, freqs, lmsts, lam, nbl, sources, positions, truths = make_peel_problem(seed=5)
    beam, beam_for = fee_peel_beam(oracle, xyzs, freqs)
    resid = simulate_residual(oracle, pc, xyzs, freqs, lmsts, lam, sources, positions, truths, beam_for)
    weights = np.ones(resid.shape[:3], np.float32)
    avg_lmst = float(np.median(lmsts))
    d_resid = dev(resid, np.float32)
    got = P.peel_timeblock(d_resid, dev(weights, np.float32), freqs, xyzs, lmsts, avg_lmst, pc, sources, positions,
                           [P.IonoConsts() for _ in sources], num_passes=2, num_loops=5, convergence=1.0,
                           freq_average_factor=4, array_latitude_rad=synth.MWA_LAT_RAD, beam="fee", fee_beam=beam)
    ref_resid, ref_consts = oracle_peel(oracle, resid, weights, pc, xyzs, freqs, lmsts, avg_lmst, sources, positions,
                                        [(0.0, 0.0, 1.0)] * len(sources), 2, 5, 1.0, 4, beam_for)
    for g, r in zip(got, ref_consts):
        assert abs(g.alpha - r[0]) <= 1e-5 * abs(r[0]) + 1e-12
        assert abs(g.beta - r[1]) <= 1e-5 * abs(r[1]) + 1e-12
        assert abs(g.gain - r[2]) <= 1e-6
    assert rel(d_resid.cpu().numpy(), ref_resid) < 1e-4


def test_batched_peel_with_fee_beam_recovers_injected_iono(oracle):
    """Both peel forms with the FEE beam recover the offsets injected through
    that beam (the batched form's shared-weights shortcut for points does not
    apply to per-tile beams)."""
    rng, pc, xyzs, freqs, lmsts, lam, nbl, sources, positions, truths = make_peel_problem(seed=7, ntiles=24, nf=16,
                                                                                           nsrc=2, points=True)
    beam, beam_for = fee_peel_beam(oracle, xyzs, freqs, seed=6)
    resid = simulate_residual(oracle, pc, xyzs, freqs, lmsts, lam, sources, positions, truths, beam_for)
    before = np.linalg.norm(resid)
    weights = np.ones(resid.shape[:3], np.float32)
    for batched in (False, True):
        d_resid = dev(resid, np.float32)
        got = P.peel_timeblock(d_resid, dev(weights, np.float32), freqs, xyzs, lmsts, float(np.median(lmsts)), pc,
                               sources, positions, [P.IonoConsts() for _ in sources], num_passes=3, num_loops=10,
                               convergence=1.0, freq_average_factor=4, array_latitude_rad=synth.MWA_LAT_RAD,
                               batched=batched, beam="fee", fee_beam=beam)
        after = np.linalg.norm(d_resid.cpu().numpy())
        for g, tr in zip(got, truths):
            assert abs(g.alpha - tr[0]) < 0.02 * abs(tr[0]) + 2e-7, (batched, g, tr)
            assert abs(g.beta - tr[1]) < 0.02 * abs(tr[1]) + 2e-7, (batched, g, tr)
            assert abs(g.gain - tr[2]) < 5e-3, (batched, g, tr)
        assert after < 0.05 * before, (batched, after, before)
