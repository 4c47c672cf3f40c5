"""Tensor-core factored point predict (tcgen05, integer byte planes, exact s32
accumulation) against the FP64 oracle.

Error metric (relative visibility error): normwise ||V - V_ref||_F / ||V_ref||_F
and the 99.9th percentile of |dV| / rms|V_ref| per visibility element.  The
bound is 1e-6 for both: the phasors enter with ~2^-24 relative error (FP32
sincospi of the FP64-reduced phase, 23-bit fixed point), X = W A with FP32
rounding and 31-bit fixed point relative to the channel's largest |W|; the
tensor-core sums themselves are exact."""

import math

import numpy as np
import pytest

from mwa_hyperdrive_b200 import srclist as sl
from mwa_hyperdrive_b200 import synth

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("no CUDA device", allow_module_level=True)

from mwa_hyperdrive_b200.model import SkyModeller  # noqa: E402

TOL = 1e-6


def errors(got, ref):
    got = np.asarray(got, np.float64)
    ref = np.asarray(ref, np.float64)
    norm = np.linalg.norm(ref)
    rms = norm / math.sqrt(ref.size)
    d = np.abs(got - ref)
    return np.linalg.norm(got - ref) / norm, np.percentile(d, 99.9) / rms, d.max() / rms


def run(sky, obs, lst, form, beam="none", f64=True):
    m = SkyModeller(sky, obs.tile_xyzs, obs.freqs, obs.phase_centre, obs.latitude, beam=beam, form=form)
    vis = torch.zeros((obs.freqs.size, obs.num_baselines, 8), dtype=torch.float64 if f64 else torch.float32,
                      device="cuda")
    m.model_timestep_with(lst, vis)
    torch.cuda.synchronize()
    return vis.cpu().numpy()


def polarised_points(n, centre, seed):
    rng = np.random.default_rng(seed)
    pos = synth.cap_positions(n, centre, math.radians(8.0), rng)
    comps = []
    for k in range(n):
        i = float(rng.lognormal(0.0, 1.0))
        fd = sl.FluxDensity(150e6, i, 0.1 * i * rng.normal(), 0.1 * i * rng.normal(), 0.05 * i * rng.normal())
        ft = [sl.PowerLaw(float(rng.normal(-0.8, 0.2)), fd),
              sl.CurvedPowerLaw(float(rng.normal(-0.8, 0.2)), fd, float(rng.normal(0, 0.2))),
              sl.FluxList([sl.FluxDensity(140e6, 2.0 * i), sl.FluxDensity(210e6, i)])][k % 3]
        comps.append(sl.SourceComponent(float(pos[k, 0]), float(pos[k, 1]), sl.Point(), ft))
    return sl.SkyModelArrays.from_components(comps)


def test_config1_tensor_vs_fp64_oracle(oracle):
    obs, sky = synth.config1()
    got = run(sky, obs, obs.lsts[0], "tensor")
    ref, _ = oracle.model_timestep(sky, obs.tile_xyzs, obs.freqs, obs.phase_centre, obs.lsts[0], obs.latitude,
                                   out_f64=True)
    nrm, p999, mx = errors(got, ref)
    print(f"config1 tensor: normwise {nrm:.2e}, p99.9 {p999:.2e}, max {mx:.2e}")
    assert nrm < TOL and p999 < TOL, (nrm, p999, mx)


@pytest.mark.parametrize("ntiles,npts,nf,beam", [(128, 1000, 6, "analytic"), (57, 77, 5, "none"), (2, 33, 3, "none"),
                                                 (128, 31, 4, "analytic")])
def test_polarised_sky_all_correlations(oracle, ntiles, npts, nf, beam):
    pc = (0.4, math.radians(-25.0))
    obs = synth.Obs(synth.tiles_in_disk(ntiles, 1000.0, ntiles), 160e6 + np.arange(nf) * 2.56e6, pc,
                    np.array([0.42]))
    sky = polarised_points(npts, pc, npts)
    got = run(sky, obs, obs.lsts[0], "tensor", beam=beam)
    b = oracle.beam_struct(1 if beam == "analytic" else 0)
    ref, _ = oracle.model_timestep(sky, obs.tile_xyzs, obs.freqs, pc, obs.lsts[0], obs.latitude, beam=b,
                                   out_f64=True)
    nrm, p999, mx = errors(got, ref)
    print(f"{ntiles} tiles {npts} comps: normwise {nrm:.2e}, p99.9 {p999:.2e}, max {mx:.2e}")
    assert nrm < TOL and p999 < TOL, (nrm, p999, mx)
    # each correlation separately (XY / YX come from the conjugate transpose)
    for k in range(4):
        r = ref[..., 2 * k:2 * k + 2]
        if np.linalg.norm(r) > 0:
            assert np.linalg.norm(got[..., 2 * k:2 * k + 2] - r) / np.linalg.norm(r) < 10 * TOL


def test_mixed_types_tensor_form_keeps_direct_gaussians_and_shapelets(oracle):
    obs, sky = synth.config2(n_points=300, n_gauss=20, n_shapelets=5, n_freqs=4, n_times=1)
    got = run(sky, obs, obs.lsts[0], "tensor", beam="analytic")
    ref, _ = oracle.model_timestep(sky, obs.tile_xyzs, obs.freqs, obs.phase_centre, obs.lsts[0], obs.latitude,
                                   beam=oracle.beam_struct(1), out_f64=True)
    nrm, p999, mx = errors(got, ref)
    assert nrm < TOL and p999 < TOL, (nrm, p999, mx)


def test_chosen_form_gaussians_and_shapelets_fp32(oracle):
    """The chosen form runs Gaussians and shapelets in the direct kernel's FP32
    form (FP32 phasor, envelope and terms; FP64 across chunks): same 1e-6 bars."""
    obs, _ = synth.config2(n_points=1, n_gauss=1, n_shapelets=1, n_freqs=5, n_times=1)
    sky = sl.SkyModelArrays.from_components(synth.gaussians_and_shapelets(60, 12, obs.phase_centre, 9))
    got = run(sky, obs, obs.lsts[0], "tensor", beam="analytic")
    ref, _ = oracle.model_timestep(sky, obs.tile_xyzs, obs.freqs, obs.phase_centre, obs.lsts[0], obs.latitude,
                                   beam=oracle.beam_struct(1), out_f64=True)
    nrm, p999, mx = errors(got, ref)
    print(f"FP32 Gaussians + shapelets: normwise {nrm:.2e}, p99.9 {p999:.2e}, max {mx:.2e}")
    assert nrm < TOL and p999 < TOL, (nrm, p999, mx)


@pytest.mark.parametrize("max_order", [5, 9])
def test_chosen_form_shapelets_dense_and_per_coefficient(oracle, max_order):
    """Shapelets alone: orders up to 5 take the dense form (basis interpolated
    once per order, dense coefficient matrix); any order of 6 or more sends
    the launch through the per-coefficient FP32 loop.  Both within 1e-6."""
    obs, _ = synth.config2(n_points=1, n_gauss=1, n_shapelets=1, n_freqs=4, n_times=1)
    rng = np.random.default_rng(17 + max_order)
    pos = synth.cap_positions(24, obs.phase_centre, math.radians(8.0), rng)
    comps = []
    for k in range(24):
        maj = math.radians(rng.uniform(0.5, 5.0) / 60.0)
        coeffs = [sl.ShapeletCoeff(int(rng.integers(0, max_order + 1)), int(rng.integers(0, max_order + 1)),
                                   float(rng.normal() * 0.1)) for _ in range(20)]
        coeffs.append(sl.ShapeletCoeff(0, 0, 1.0))
        comps.append(sl.SourceComponent(float(pos[k, 0]), float(pos[k, 1]),
                                        sl.Shapelet(maj, maj * rng.uniform(0.3, 1.0), rng.uniform(0, math.pi), coeffs),
                                        sl.PowerLaw(-0.8, sl.FluxDensity(150e6, float(rng.lognormal()), 0.0, 0.0, 0.0))))
    sky = sl.SkyModelArrays.from_components(comps)
    got = run(sky, obs, obs.lsts[0], "tensor", beam="analytic")
    ref, _ = oracle.model_timestep(sky, obs.tile_xyzs, obs.freqs, obs.phase_centre, obs.lsts[0], obs.latitude,
                                   beam=oracle.beam_struct(1), out_f64=True)
    nrm, p999, mx = errors(got, ref)
    print(f"shapelets to order {max_order}: normwise {nrm:.2e}, p99.9 {p999:.2e}, max {mx:.2e}")
    assert nrm < TOL and p999 < TOL, (nrm, p999, mx)


@pytest.mark.parametrize("ntiles,npts", [(64, 4500), (24, 16500), (97, 3000)])
def test_many_components(oracle, ntiles, npts):
    """Errors must not grow with the component count; 16500 components need
    two launches (16384 + 116) that accumulate in turn."""
    pc = (0.1, math.radians(-30.0))
    obs = synth.Obs(synth.tiles_in_disk(ntiles, 1000.0, 7), 180e6 + np.arange(2) * 1.28e6, pc, np.array([0.15]))
    sky = polarised_points(npts, pc, 11)
    got = run(sky, obs, obs.lsts[0], "tensor")
    ref, _ = oracle.model_timestep(sky, obs.tile_xyzs, obs.freqs, pc, obs.lsts[0], obs.latitude, out_f64=True)
    nrm, p999, mx = errors(got, ref)
    print(f"{npts} comps: normwise {nrm:.2e}, p99.9 {p999:.2e}, max {mx:.2e}")
    assert nrm < TOL and p999 < TOL, (nrm, p999, mx)


def test_bright_source_over_faint_field(oracle):
    """Flux spanning 1e-4 .. 1e2 Jy: x is fixed point relative to the brightest
    component, which the faint ones must survive."""
    pc = (0.3, math.radians(-20.0))
    rng = np.random.default_rng(5)
    pos = synth.cap_positions(600, pc, math.radians(10.0), rng)
    comps = []
    for k in range(600):
        i = 100.0 if k == 0 else float(10.0 ** rng.uniform(-4.0, 0.0))
        comps.append(sl.SourceComponent(float(pos[k, 0]), float(pos[k, 1]), sl.Point(),
                                        sl.PowerLaw(-0.7, sl.FluxDensity(150e6, i, 0.02 * i, 0.0, 0.0))))
    sky = sl.SkyModelArrays.from_components(comps)
    obs = synth.Obs(synth.tiles_in_disk(128, 1500.0, 3), 150e6 + np.arange(3) * 5e6, pc, np.array([0.31]))
    got = run(sky, obs, obs.lsts[0], "tensor", beam="analytic")
    ref, _ = oracle.model_timestep(sky, obs.tile_xyzs, obs.freqs, pc, obs.lsts[0], obs.latitude,
                                   beam=oracle.beam_struct(1), out_f64=True)
    nrm, p999, mx = errors(got, ref)
    print(f"bright + faint: normwise {nrm:.2e}, p99.9 {p999:.2e}, max {mx:.2e}")
    assert nrm < TOL and p999 < TOL, (nrm, p999, mx)
    # the faint field alone (bright source subtracted in FP64 on both sides) is still right
    bright = sl.SkyModelArrays.from_components(comps[:1])
    got_b = run(bright, obs, obs.lsts[0], "direct", beam="analytic")
    ref_b, _ = oracle.model_timestep(bright, obs.tile_xyzs, obs.freqs, pc, obs.lsts[0], obs.latitude,
                                     beam=oracle.beam_struct(1), out_f64=True)
    faint_ref = ref - ref_b
    faint_got = got - got_b
    rel = np.linalg.norm(faint_got - faint_ref) / np.linalg.norm(faint_ref)
    print(f"faint field relative error {rel:.2e}")
    assert rel < 1e-4


def test_f32_output_and_accumulate(oracle):
    obs, sky = synth.config1()
    obs.freqs = obs.freqs[:3]
    m = SkyModeller(sky, obs.tile_xyzs, obs.freqs, obs.phase_centre, obs.latitude, form="tensor")
    vis = torch.ones((3, obs.num_baselines, 8), dtype=torch.float32, device="cuda")
    m.model_timestep_with(obs.lsts[0], vis)
    torch.cuda.synchronize()
    ref, _ = oracle.model_timestep(sky, obs.tile_xyzs, obs.freqs, obs.phase_centre, obs.lsts[0], obs.latitude,
                                   out_f64=True)
    nrm, p999, _ = errors(vis.cpu().numpy() - 1.0, ref)
    assert nrm < 5e-6  # f32 output rounding dominates


@pytest.mark.parametrize("ctype,name", [(0, "points"), (1, "Gaussians"), (2, "shapelets")])
def test_full_mixed_config_chosen_form_vs_fp64_oracle(oracle, ctype, name):
    """The timed configuration itself: 128 tiles, all 4 timesteps and 384
    channels, 4000 points / 500 Gaussians / 100 shapelets (20 coefficients)
    through the analytic beam, each class predicted by the chosen form
    (tensor-core points, FP32-form Gaussians and shapelets) with the f32
    output the benchmark times, against the FP64 oracle on a seeded sample
    of 276 baselines (every baseline among 24 random tiles) at every
    (timestep, channel).  Bars: normwise and p99.9 below 1e-6."""
    obs, sky = synth.config2()
    cls = sky.select(sky.comp_type == ctype)
    sub, bl = synth.sample_tiles(obs.num_tiles, 24, 2024)
    m = SkyModeller(cls, obs.tile_xyzs, obs.freqs, obs.phase_centre, obs.latitude, beam="analytic", form="tensor")
    vis = torch.zeros((obs.freqs.size, obs.num_baselines, 8), dtype=torch.float32, device="cuda")
    idx = torch.from_numpy(bl).cuda()
    got, ref = [], []
    for t, lst in enumerate(obs.lsts):
        vis.zero_()
        m.model_timestep_with(float(lst), vis, return_uvws=False)
        got.append(vis.index_select(1, idx).cpu().numpy())
        r, _ = oracle.model_timestep(cls, obs.tile_xyzs[sub], obs.freqs, obs.phase_centre, float(lst), obs.latitude,
                                     beam=oracle.beam_struct(1), out_f64=True)
        ref.append(r)
    m.close()
    nrm, p999, mx = errors(np.stack(got), np.stack(ref))
    print(f"config 2 {name} ({cls.num_components}), 4 x 384 x 276 sampled: normwise {nrm:.2e}, p99.9 {p999:.2e}, "
          f"max {mx:.2e}")
    assert nrm < TOL and p999 < TOL, (nrm, p999, mx)


def host_buffer_matches_device(m, obs, lst):
    dev = torch.zeros((obs.freqs.size, obs.num_baselines, 8), dtype=torch.float32, device="cuda")
    m.model_timestep_with(lst, dev, return_uvws=False)
    want = dev.cpu().numpy()
    host = np.zeros((obs.freqs.size, obs.num_baselines, 8), np.float32)
    m.model_timestep_with_host(lst, host)
    np.testing.assert_array_equal(host, want)
    # accumulation into what the buffer held: the additions' order differs
    # from the device call's, so equal to FP32 rounding at the visibilities'
    # scale (2 ulp of the largest magnitude)
    host = np.full((obs.freqs.size, obs.num_baselines, 8), 0.5, np.float32)
    m.model_timestep_with_host(lst, host)
    tol = 2 * float(np.spacing(np.float32(np.abs(want).max())))
    # a masked pol is zero after either call, the buffer's 0.5 included
    masked = np.all(want == 0, axis=(0, 1))
    np.testing.assert_allclose(host, np.where(masked, np.float32(0), want + np.float32(0.5)), rtol=0, atol=tol)


def test_host_buffer_call_equals_device_call():
    """The trait's host-buffer call -- the Gaussians and shapelets of every
    channel staged while the buffer uploads, then the points chunk by chunk
    with each chunk's download behind them -- accumulates exactly the device
    call's visibilities into the caller's buffer (the timed configuration,
    one timestep, every component class)."""
    obs, sky = synth.config2()
    m = SkyModeller(sky, obs.tile_xyzs, obs.freqs, obs.phase_centre, obs.latitude, beam="analytic", form="tensor")
    host_buffer_matches_device(m, obs, float(obs.lsts[1]))
    m.close()


@pytest.mark.parametrize("pols,ng,ns", [("XX_YY", 60, 0), ("XX", 0, 12), ("XX_YY_XY", 30, 6), ("XX_XY_YX_YY", 0, 0)])
def test_host_buffer_call_chunks_and_masks(pols, ng, ns):
    """The same at 160 channels (three tables of points: 74 + 74 + 12
    channels, each downloaded behind its own Gram products) for points with
    Gaussians, with shapelets, with both, and alone (the five-chunk pipeline
    of the other forms), under every pol mask."""
    obs, sky = synth.config2(n_gauss=ng, n_shapelets=ns, n_freqs=160, n_times=1)
    m = SkyModeller(sky, obs.tile_xyzs, obs.freqs, obs.phase_centre, obs.latitude, pols=pols, beam="analytic",
                    form="tensor")
    host_buffer_matches_device(m, obs, float(obs.lsts[0]))
    m.close()


@pytest.mark.parametrize("ntiles,npts", [(130, 200), (144, 300), (256, 150), (300, 64)])
def test_more_than_128_tiles(oracle, ntiles, npts):
    """Any tile count: the products run in blocks of 128 rows x 64 columns
    (XX and YY only the blocks that hold a baseline p < q); every baseline is
    written once through the planar epilogue."""
    pc = (0.2, math.radians(-26.0))
    obs = synth.Obs(synth.tiles_in_disk(ntiles, 1500.0, ntiles), 170e6 + np.arange(3) * 1.28e6, pc,
                    np.array([0.25]))
    sky = polarised_points(npts, pc, ntiles + 1)
    got = run(sky, obs, obs.lsts[0], "tensor", beam="analytic")
    ref, _ = oracle.model_timestep(sky, obs.tile_xyzs, obs.freqs, pc, obs.lsts[0], obs.latitude,
                                   beam=oracle.beam_struct(1), out_f64=True)
    nrm, p999, mx = errors(got, ref)
    print(f"{ntiles} tiles: normwise {nrm:.2e}, p99.9 {p999:.2e}, max {mx:.2e}")
    assert nrm < TOL and p999 < TOL, (nrm, p999, mx)


@pytest.mark.parametrize("ntiles,npts", [(144, 200), (256, 120)])
def test_per_tile_beams_tensor_form(oracle, ntiles, npts):
    """Per-tile beams in the tensor form (block form over twice the
    components) past 128 tiles, with Gaussians in the same sky (the chosen
    form's per-tile kernel up to 32 unique beams, here 18 and 30): against
    the oracle with the same explicit per-tile Jones table, within 1e-6."""
    pc = (0.2, math.radians(-26.0))
    obs = synth.Obs(synth.tiles_in_disk(ntiles, 1500.0, ntiles + 3), 166.4e6 + np.arange(3) * 0.96e6, pc,
                    np.array([0.3]))
    sky = polarised_points(npts, pc, ntiles + 5)
    comps = [sl.SourceComponent(float(sky.ra[k]), float(sky.dec[k]), sl.Point(),
                                sl.PowerLaw(float(sky.si[k]), sl.FluxDensity(*sky.fds[sky.fd_start[k]])))
             for k in range(npts) if sky.flux_type[k] == 1]
    comps += synth.gaussians_and_shapelets(10, 0, pc, 6)
    sky = sl.SkyModelArrays.from_components(comps)
    rng = np.random.default_rng(ntiles)
    gains = np.ones((ntiles, 2, 16))
    for p in rng.choice(ntiles, ntiles // 4, replace=False):
        gains[p, rng.integers(2), rng.integers(16)] = 0.0
    m = SkyModeller(sky, obs.tile_xyzs, obs.freqs, pc, obs.latitude, beam="per_tile", dipole_gains=gains,
                    form="tensor")
    vis = torch.zeros((obs.freqs.size, obs.num_baselines, 8), dtype=torch.float64, device="cuda")
    m.model_timestep_with(obs.lsts[0], vis)
    torch.cuda.synchronize()
    uniq, tmap, ufreqs, fmap = oracle.unique_tile_beams(gains, obs.freqs)
    tabs = [oracle.tile_beam_table(sky, ty, obs.lsts[0], obs.latitude, uniq, ufreqs) if ty < 2 else None
            for ty in range(3)]
    ref, _ = oracle.model_timestep(sky, obs.tile_xyzs, obs.freqs, pc, obs.lsts[0], obs.latitude,
                                   beam=oracle.beam_struct(2, tabs, tmap, fmap, ufreqs.size), out_f64=True)
    nrm, p999, mx = errors(vis.cpu().numpy(), ref)
    print(f"per-tile beams {ntiles} tiles, {len(uniq)} beams: normwise {nrm:.2e}, p99.9 {p999:.2e}, max {mx:.2e}")
    assert nrm < TOL and p999 < TOL, (nrm, p999, mx)


@pytest.mark.parametrize("ctype", [1, 2])
def test_chosen_form_per_tile_beams_gaussians_and_shapelets(oracle, ctype):
    """With a beam per tile and at most 32 unique tiles, the chosen form's
    Gaussians and shapelets run in the per-tile kernel of the chosen form
    (FP32 phasor and envelope; G = B_p S and H = B_q staged per chunk, the
    products in FP64): against the oracle with the same explicit per-tile
    Jones table within 1e-6, and not the FP64 per-tile kernel's result (a
    different kernel ran)."""
    pc = (0.2, math.radians(-26.0))
    obs = synth.Obs(synth.tiles_in_disk(48, 1500.0, 7), 166.4e6 + np.arange(5) * 0.64e6, pc, np.array([0.3]))
    comps = synth.gaussians_and_shapelets(60 if ctype == 1 else 0, 0 if ctype == 1 else 12, pc, 8)
    sky = sl.SkyModelArrays.from_components(comps)
    rng = np.random.default_rng(3)
    gains = np.ones((obs.num_tiles, 2, 16))
    for p in rng.choice(obs.num_tiles, 12, replace=False):
        gains[p, rng.integers(2), rng.integers(16)] = 0.0
    out = {}
    for form in ("tensor", "direct"):
        m = SkyModeller(sky, obs.tile_xyzs, obs.freqs, pc, obs.latitude, beam="per_tile", dipole_gains=gains,
                        form=form)
        vis = torch.zeros((obs.freqs.size, obs.num_baselines, 8), dtype=torch.float64, device="cuda")
        m.model_timestep_with(obs.lsts[0], vis)
        torch.cuda.synchronize()
        out[form] = vis.cpu().numpy()
    uniq, tmap, ufreqs, fmap = oracle.unique_tile_beams(gains, obs.freqs)
    assert 2 < len(uniq) <= 32
    tabs = [oracle.tile_beam_table(sky, ty, obs.lsts[0], obs.latitude, uniq, ufreqs) if ty == ctype else None
            for ty in range(3)]
    ref, _ = oracle.model_timestep(sky, obs.tile_xyzs, obs.freqs, pc, obs.lsts[0], obs.latitude,
                                   beam=oracle.beam_struct(2, tabs, tmap, fmap, ufreqs.size), out_f64=True)
    nrm, p999, mx = errors(out["tensor"], ref)
    print(f"per-tile chosen form, type {ctype}, {len(uniq)} beams: normwise {nrm:.2e}, p99.9 {p999:.2e}, max {mx:.2e}")
    assert nrm < TOL and p999 < TOL, (nrm, p999, mx)
    assert errors(out["direct"], ref)[0] < 1e-10
    assert errors(out["tensor"], out["direct"])[0] > 1e-12
