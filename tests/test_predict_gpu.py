"""Predictor parity on the GPU: libhdc's CUDA kernels (through the C ABI)
against the CPU oracle.

Tolerances: FP64 output mode within 1e-10 relative (normwise, and per
visibility relative to the rms visibility); the reference-style f32 output
within 2 f32 ulps of the oracle's identically demoted result.
"""

import ctypes
import json
import math
from pathlib import Path

import numpy as np
import pytest

from mwa_hyperdrive_b200 import srclist as sl
from mwa_hyperdrive_b200 import synth

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("no CUDA device", allow_module_level=True)

from mwa_hyperdrive_b200 import _lib  # noqa: E402
from mwa_hyperdrive_b200.model import SkyModeller  # noqa: E402

GOLD = Path(__file__).resolve().parent / "golden"
KATS = json.loads((GOLD / "model_kats.json").read_text())
LAT = synth.MWA_LAT_RAD


def rel_err(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    norm = np.linalg.norm(b)
    rms = norm / math.sqrt(max(b.size, 1))
    return np.linalg.norm(a - b) / max(norm, 1e-300), np.max(np.abs(a - b)) / max(rms, 1e-300)


def assert_f32_close(a, b, ulps=2):
    a = np.asarray(a, np.float32)
    b = np.asarray(b, np.float32)
    scale = np.maximum(np.abs(b), np.float32(np.max(np.abs(b)) * 1e-6 + 1e-30))
    tol = ulps * np.spacing(scale)
    bad = np.abs(a - b) > tol
    assert not bad.any(), f"{bad.sum()} elements differ by more than {ulps} ulp; max diff {np.max(np.abs(a - b))}"


def dev(x):
    return torch.from_numpy(np.ascontiguousarray(x)).cuda()


def run_modeller(sky, obs, lst, f64=True, beam="none", pols="XX_XY_YX_YY", form="direct"):
    m = SkyModeller(sky, obs.tile_xyzs, obs.freqs, obs.phase_centre, obs.latitude, pols=pols, beam=beam, form=form)
    vis = torch.zeros((obs.freqs.size, obs.num_baselines, 8), dtype=torch.float64 if f64 else torch.float32,
                      device="cuda")
    uvws = m.model_timestep_with(lst, vis)
    torch.cuda.synchronize()
    return vis.cpu().numpy(), uvws, m


# ---------------------------------------------------------------- KATs
def kat_obs():
    o = KATS["obs"]
    pc = tuple(math.radians(x) for x in o["phase_centre_deg"])
    return synth.Obs(np.array(o["xyzs"], np.float64), np.array(o["freqs_hz"]), pc, np.array([0.0]))


def kat_comp(kind, pos, ctype):
    flux = {"list": sl.FluxList([sl.FluxDensity(150e6, 1.0), sl.FluxDensity(175e6, 3.0), sl.FluxDensity(200e6, 2.0)]),
            "power_law": sl.PowerLaw(-0.8, sl.FluxDensity(150e6, 1.0)),
            "curved_power_law": sl.CurvedPowerLaw(-0.8, sl.FluxDensity(150e6, 1.0), 0.03)}[kind]
    t = [sl.Point(), sl.Gaussian(0.0, 0.0, 0.0), sl.Shapelet(0.0, 0.0, 0.0, [sl.ShapeletCoeff(0, 0, 1.0)])][ctype]
    return sl.SourceComponent(*sl.radec_deg(*pos), t, flux)


KCASES = [("list", (0.0, -27.0), "test_list_zenith_visibilities"),
          ("power_law", (0.0, -27.0), "test_power_law_zenith_visibilities"),
          ("curved_power_law", (0.0, -27.0), "test_curved_power_law_zenith_visibilities"),
          ("list", (1.0, -27.0), "test_list_off_zenith_visibilities"),
          ("power_law", (1.0, -27.0), "test_power_law_off_zenith_visibilities"),
          ("curved_power_law", (1.0, -27.0), "test_curved_power_law_off_zenith_visibilities")]


@pytest.mark.parametrize("ctype", [0, 1, 2])
@pytest.mark.parametrize("kind,pos,name", KCASES)
def test_kats_native_modeller(ctype, kind, pos, name):
    obs = kat_obs()
    sky = sl.SkyModelArrays.from_components([kat_comp(kind, pos, ctype)])
    vis, uvws, _ = run_modeller(sky, obs, 0.0, f64=False)
    gold = np.array(KATS["cases"][name], np.float32).reshape(3, 3, 8)
    assert_f32_close(vis, gold, ulps=1)


@pytest.mark.parametrize("ctype,name", [(1, "test_multiple_gaussian_components"),
                                        (2, "test_multiple_shapelet_components")])
def test_kats_multiple_components(ctype, name):
    obs = kat_obs()
    sky = sl.SkyModelArrays.from_components([kat_comp("list", (1.0, -27.0), ctype),
                                             kat_comp("list", (1.1, -27.0), ctype)])
    vis, _, _ = run_modeller(sky, obs, 0.0, f64=False)
    assert_f32_close(vis, np.array(KATS["cases"][name], np.float32).reshape(3, 3, 8), ulps=1)


# ------------------------------------------------------- config-1 parity
def test_config1_f64_parity(oracle):
    obs, sky = synth.config1()
    vis, uvws, _ = run_modeller(sky, obs, obs.lsts[0], f64=True)
    ref, ref_uvws = oracle.model_timestep(sky, obs.tile_xyzs, obs.freqs, obs.phase_centre, obs.lsts[0], LAT,
                                          out_f64=True)
    np.testing.assert_allclose(uvws, ref_uvws, rtol=0, atol=1e-9)
    nrm, mx = rel_err(vis, ref)
    assert nrm < 1e-10 and mx < 1e-10, (nrm, mx)


def test_config1_f32_mode(oracle):
    obs, sky = synth.config1()
    vis, _, _ = run_modeller(sky, obs, obs.lsts[0], f64=False)
    ref, _ = oracle.model_timestep(sky, obs.tile_xyzs, obs.freqs, obs.phase_centre, obs.lsts[0], LAT)
    assert_f32_close(vis, ref, ulps=2)


def small_obs(ntiles=23, nf=7, seed=5):
    pc = (0.3, math.radians(-30.0))
    return synth.Obs(synth.tiles_in_disk(ntiles, 1500.0, seed), 160e6 + np.arange(nf) * 1.28e6, pc,
                     np.array([0.3 + 0.01]))


def mixed_sky(seed=3, npts=70, ng=33, ns=9):
    rng = np.random.default_rng(seed)
    pc = (0.3, math.radians(-30.0))
    comps = synth.point_sky(npts, pc, 8.0, seed, curved_q_sigma=0.2)
    comps += synth.gaussians_and_shapelets(ng, ns, pc, seed + 1)
    # a few list-flux components of each type
    pos = synth.cap_positions(6, pc, math.radians(5.0), rng)
    for k in range(6):
        fl = sl.FluxList([sl.FluxDensity(120e6, 2.0 + k), sl.FluxDensity(170e6, 1.5), sl.FluxDensity(200e6, -0.3)])
        t = [sl.Point(), sl.Gaussian(1e-3, 5e-4, 0.4),
             sl.Shapelet(1e-3, 6e-4, 1.1, [sl.ShapeletCoeff(1, 2, 0.3), sl.ShapeletCoeff(0, 0, 1.0)])][k % 3]
        comps.append(sl.SourceComponent(float(pos[k, 0]), float(pos[k, 1]), t, fl))
    return sl.SkyModelArrays.from_components(comps)


@pytest.mark.parametrize("beam", ["none", "analytic"])
def test_mixed_types_f64_parity(oracle, beam):
    obs = small_obs()
    sky = mixed_sky()
    lst = obs.lsts[0]
    vis, _, _ = run_modeller(sky, obs, lst, f64=True, beam=beam)
    b = oracle.beam_struct(1 if beam == "analytic" else 0)
    ref, _ = oracle.model_timestep(sky, obs.tile_xyzs, obs.freqs, obs.phase_centre, lst, LAT, beam=b, out_f64=True)
    nrm, mx = rel_err(vis, ref)
    assert nrm < 1e-10 and mx < 1e-10, (nrm, mx)


@pytest.mark.parametrize("pols", ["XX", "YY", "XX_YY", "XX_YY_XY"])
def test_pols_mask(oracle, pols):
    obs = small_obs(9, 3)
    sky = mixed_sky(npts=5, ng=2, ns=1)
    vis, _, _ = run_modeller(sky, obs, obs.lsts[0], f64=False, pols=pols, beam="analytic")
    code = {"XX": 1, "YY": 2, "XX_YY": 3, "XX_YY_XY": 4}[pols]
    ref, _ = oracle.model_timestep(sky, obs.tile_xyzs, obs.freqs, obs.phase_centre, obs.lsts[0], LAT,
                                   beam=oracle.beam_struct(1), pols=code)
    assert_f32_close(vis, ref, ulps=2)


def test_edge_shapes(oracle):
    # 2 tiles (one baseline), 1 channel; component counts around the chunk size
    for ntiles, npts in [(2, 1), (3, 64), (17, 65), (40, 129)]:
        obs = small_obs(ntiles, 1, seed=ntiles)
        sky = sl.SkyModelArrays.from_components(synth.point_sky(npts, obs.phase_centre, 5.0, npts))
        vis, _, _ = run_modeller(sky, obs, obs.lsts[0], f64=True)
        ref, _ = oracle.model_timestep(sky, obs.tile_xyzs, obs.freqs, obs.phase_centre, obs.lsts[0], LAT,
                                       out_f64=True)
        nrm, mx = rel_err(vis, ref)
        assert nrm < 1e-10 and mx < 1e-10, (ntiles, npts, nrm, mx)


def test_empty_sky_and_accumulate(oracle):
    obs = small_obs(5, 2)
    empty = sl.SkyModelArrays.from_components([])
    m = SkyModeller(empty, obs.tile_xyzs, obs.freqs, obs.phase_centre, LAT)
    vis = torch.full((2, 10, 8), 1.5, dtype=torch.float32, device="cuda")
    m.model_timestep_with(obs.lsts[0], vis)
    assert torch.all(vis == 1.5)
    # accumulation (+=) semantics
    sky = mixed_sky(npts=4, ng=1, ns=1)
    m2 = SkyModeller(sky, obs.tile_xyzs, obs.freqs, obs.phase_centre, LAT)
    v64 = torch.zeros((2, 10, 8), dtype=torch.float64, device="cuda")
    m2.model_timestep_with(obs.lsts[0], v64)
    m2.model_timestep_with(obs.lsts[0], v64)
    ref, _ = oracle.model_timestep(sky, obs.tile_xyzs, obs.freqs, obs.phase_centre, obs.lsts[0], LAT, out_f64=True)
    nrm, _ = rel_err(v64.cpu().numpy(), 2 * ref)
    assert nrm < 1e-10


def test_host_buffer_call_and_autos(oracle):
    obs = small_obs(11, 4)
    sky = mixed_sky(npts=12, ng=3, ns=2)
    m = SkyModeller(sky, obs.tile_xyzs, obs.freqs, obs.phase_centre, LAT, beam="analytic")
    vis, uvws = m.model_timestep(obs.lsts[0])
    ref, ref_uvws = oracle.model_timestep(sky, obs.tile_xyzs, obs.freqs, obs.phase_centre, obs.lsts[0], LAT,
                                          beam=oracle.beam_struct(1))
    assert_f32_close(vis, ref, ulps=2)
    autos = torch.zeros((4, 11, 8), dtype=torch.float32, device="cuda")
    m.model_timestep_autos_with(obs.lsts[0], autos)
    ref_a = oracle.model_autos(sky, 11, obs.freqs, obs.lsts[0], LAT, beam=oracle.beam_struct(1))
    assert_f32_close(autos.cpu().numpy(), ref_a, ulps=2)


def test_update_with_a_source(oracle):
    obs = small_obs(9, 3)
    sky = mixed_sky(npts=6, ng=2, ns=1)
    m = SkyModeller(sky, obs.tile_xyzs, obs.freqs, obs.phase_centre, LAT)
    src = mixed_sky(seed=9, npts=3, ng=1, ns=1)
    new_pc = (0.31, math.radians(-29.0))
    m.update_with_a_source(src, new_pc)
    vis = torch.zeros((3, 36, 8), dtype=torch.float64, device="cuda")
    m.model_timestep_with(obs.lsts[0], vis)
    ref, _ = oracle.model_timestep(src, obs.tile_xyzs, obs.freqs, new_pc, obs.lsts[0], LAT, out_f64=True)
    nrm, mx = rel_err(vis.cpu().numpy(), ref)
    assert nrm < 1e-10 and mx < 1e-10


def test_shapelet_index_clamp_far_baselines(oracle):
    # baselines long enough that the basis position leaves the table on both
    # sides: the kernel must clamp (and match the oracle's clamp) without
    # reading outside the table.
    pc = (0.0, math.radians(-27.0))
    xyzs = synth.enu_to_xyz(np.array([0.0, 6.0e4, -6.0e4]), np.array([0.0, 3.0e4, -5.0e4]), np.zeros(3))
    obs = synth.Obs(xyzs, np.array([200e6]), pc, np.array([0.0]))
    comp = sl.SourceComponent(0.01, math.radians(-27.2), sl.Shapelet(0.02, 0.01, 0.3, [sl.ShapeletCoeff(2, 1, 1.0)]),
                              sl.PowerLaw(-0.7, sl.FluxDensity(150e6, 3.0)))
    sky = sl.SkyModelArrays.from_components([comp])
    vis, _, _ = run_modeller(sky, obs, 0.0, f64=True)
    ref, _ = oracle.model_timestep(sky, xyzs, obs.freqs, pc, 0.0, LAT, out_f64=True)
    np.testing.assert_allclose(vis, ref, rtol=1e-10, atol=1e-12)


# ------------------------------------------------------- drop-in layer
def _rime_tables(sky_arr, obs, beam_tiles=None, seed=0):
    """Build the reference's device tables (gpu/types.h) for one component
    type from a sky model whose power laws are referenced at 150 MHz."""
    import mwa_hyperdrive_b200.srclist as S

    from oracle import oracle as orc

    n = sky_arr.num_components
    groups = {1: [], 2: [], 0: []}
    for k in range(n):
        groups[int(sky_arr.flux_type[k])].append(k)
    order = groups[1] + groups[2] + groups[0]
    lmn = np.array([orc.lmn_rime(sky_arr.ra[k], sky_arr.dec[k], *obs.phase_centre) for k in order]).reshape(-1, 3)
    inst150 = orc.inst_flux(sky_arr, [150e6])[0]  # [nc][8]
    return order, groups, lmn, inst150


@pytest.mark.parametrize("ctype", [0, 1, 2])
@pytest.mark.parametrize("fee", [False, True])
def test_dropin_model_functions_per_tile_beam(oracle, ctype, fee):
    """The drop-in model_* with a per-tile beam table [uniq tile][uniq freq]
    [component] and its maps: a random table, or (fee) the reference's own
    flow, where BeamGpu::calc_jones_pair fills the table and the Addresses
    carry the beam's device tile and frequency maps (model/gpu.rs:889-910),
    here hdc_fee_calc_jones and hdc_fee_beam_tile_map / _freq_map."""
    obs = small_obs(12, 5)
    rng = np.random.default_rng(11 + ctype)
    pc = obs.phase_centre
    comps = []
    pos = synth.cap_positions(9, pc, math.radians(6.0), rng)
    for k in range(9):
        fd = sl.FluxDensity(150e6, float(rng.uniform(0.5, 3.0)), 0.1, -0.05, 0.02)
        ft = [sl.PowerLaw(-0.7, fd), sl.CurvedPowerLaw(-0.9, fd, 0.1),
              sl.FluxList([sl.FluxDensity(140e6, 2.0), sl.FluxDensity(190e6, 1.0)])][k % 3]
        t = [sl.Point(), sl.Gaussian(2e-3, 1e-3, 0.7),
             sl.Shapelet(2e-3, 1e-3, 0.7, [sl.ShapeletCoeff(1, 0, 0.5), sl.ShapeletCoeff(2, 3, -0.2)])][ctype]
        comps.append(sl.SourceComponent(float(pos[k, 0]), float(pos[k, 1]), t, ft))
    # the reference's GPU component order: power laws, curved, lists
    comps = [comps[i] for i in range(0, 9, 3)] + [comps[i] for i in range(1, 9, 3)] + [comps[i] for i in range(2, 9, 3)]
    sky = sl.SkyModelArrays.from_components(comps)
    nf, nbl, nt = obs.freqs.size, obs.num_baselines, obs.num_tiles
    lst = obs.lsts[0]
    uvws = oracle.xyzs_to_cross_uvws(obs.tile_xyzs, lst - pc[0], pc[1])
    # per-tile beam: 3 unique tiles, 2 unique freqs
    tile_map = (np.arange(nt) % 3).astype(np.int32)
    freq_map = (np.arange(nf) * 2 // nf).astype(np.int32)
    beam = (rng.normal(size=(3, 2, 9, 8)) * 0.3)
    beam[..., 0] += 1.0
    beam[..., 6] += 1.0
    n_uniq_freq = 2
    if fee:
        from mwa_hyperdrive_b200.fee import FeeBeam

        delays = np.tile(np.arange(16, dtype=np.uint32) % 4, (nt, 1))
        delays[1, 3] = delays[4, 9] = 32  # dead dipoles: three unique tiles
        fb = FeeBeam(synth.fee_coeffs([160000000, 161280000, 162560000, 163840000], 7, seed=2), obs.freqs, delays,
                     np.ones((nt, 32)))
        tile_map, freq_map = fb.maps()
        n_uniq_freq = fb.num_unique_freqs()
        azza = [oracle.hadec_to_azel(lst - c.ra, c.dec, LAT) for c in comps]
        az = np.array([a for a, _ in azza])
        za = np.array([math.pi / 2 - e for _, e in azza])
        beam = fb.calc_jones(az, za, latitude_rad=LAT).cpu().numpy()
    lmn = np.array([oracle.lmn_rime(c.ra, c.dec, *pc) for c in comps])
    inst150 = oracle.inst_flux(sky, [150e6])[0]
    list_fds = oracle.inst_flux(sky, obs.freqs)[:, 6:9]  # [nf][3][8]
    d = {}

    def put(name, arr, dt=np.float64):
        d[name] = dev(np.ascontiguousarray(arr, dt))
        return d[name].data_ptr()

    lm = put("lmn", lmn)
    fds = put("fds", inst150)
    sis = put("sis", np.array([-0.7] * 3 + [-0.9] * 3))
    qs = put("qs", np.array([0.1] * 3))
    lf = put("lf", list_fds)
    gpar = put("gp", np.array([[2e-3, 1e-3, 0.7]] * 9))
    suv = oracle.shapelet_uvws(sky, obs.tile_xyzs, lst)[..., :2]  # [bl][9][2]
    suv_pl = put("suv_pl", suv[:, 0:3])
    suv_cpl = put("suv_cpl", suv[:, 3:6])
    suv_l = put("suv_l", suv[:, 6:9])
    coeff_dt = np.dtype([("value", np.float64), ("n1", np.uint8), ("n2", np.uint8), ("pad", np.uint8, 6)])
    co = np.zeros(2, coeff_dt)
    co["value"] = [0.5, -0.2]
    co["n1"] = [1, 2]
    co["n2"] = [0, 3]
    co3 = np.concatenate([co] * 9)  # 3 groups x 3 components x 2 coefficients
    coeffs = put("co", co3.view(np.uint8), np.uint8)
    ncoef = put("nco", np.array([2] * 9, np.int32), np.int32)
    freqs = put("freqs", obs.freqs)
    tm = put("tm", tile_map, np.int32)
    fm = put("fm", freq_map, np.int32)
    um = put("um", np.arange(nt, dtype=np.int32), np.int32)
    bj = put("beam", beam)
    d_uvws = put("uvws", uvws)
    vis = torch.zeros((nf, nbl, 8), dtype=torch.float32, device="cuda")
    if fee:  # the beam's own device maps, as the reference's Addresses carry them
        tm, fm = _lib.lib().hdc_fee_beam_tile_map(fb.handle), _lib.lib().hdc_fee_beam_freq_map(fb.handle)
    a = _lib.Addresses(nf, nf * nbl, nbl, freqs, 0, n_uniq_freq, tm, fm, um)
    L = _lib.lib()
    o3 = lambda off: lm + off * 24  # noqa: E731
    if ctype == 0:
        p = _lib.Points(3, o3(0), fds, sis, 3, o3(3), fds + 3 * 64, sis + 3 * 8, qs, 3, o3(6), lf)
        res = L.model_points(ctypes.byref(p), ctypes.byref(a), d_uvws, bj, vis.data_ptr())
    elif ctype == 1:
        p = _lib.Gaussians(3, o3(0), fds, sis, gpar, 3, o3(3), fds + 3 * 64, sis + 3 * 8, qs, gpar + 72, 3, o3(6), lf,
                           gpar + 144)
        res = L.model_gaussians(ctypes.byref(p), ctypes.byref(a), d_uvws, bj, vis.data_ptr())
    else:
        p = _lib.Shapelets(3, o3(0), fds, sis, gpar, suv_pl, coeffs, ncoef,
                           3, o3(3), fds + 3 * 64, sis + 3 * 8, qs, gpar + 72, suv_cpl, coeffs + 96, ncoef + 12,
                           3, o3(6), lf, gpar + 144, suv_l, coeffs + 192, ncoef + 24)
        res = L.model_shapelets(ctypes.byref(p), ctypes.byref(a), d_uvws, bj, vis.data_ptr())
    _lib.check_str(res, "model_*")
    torch.cuda.synchronize()
    # oracle with the explicit per-tile beam
    bj_t = [None, None, None]
    bj_t[ctype] = beam
    b = oracle.beam_struct(2, bj_t, tile_map, freq_map, n_uniq_freq)
    ref = oracle.model_type(ctype, sky, obs.tile_xyzs, obs.freqs, pc, lst, LAT, uvws, beam=b)
    assert_f32_close(vis.cpu().numpy(), ref, ulps=4)


# ---------------------------------------------------------- per-tile beams
def dipole_gains(ntiles, seed, damaged=0.3):
    """[tile][2][16] dipole amplitudes: most tiles intact, a fraction with one
    or two dead dipoles (a few distinct patterns, so tiles share beams)."""
    rng = np.random.default_rng(seed)
    g = np.ones((ntiles, 2, 16))
    patterns = [(0, 5), (1, 12), (0, 3), (1, 0)]
    for p in range(ntiles):
        if rng.random() < damaged:
            pol, d = patterns[rng.integers(len(patterns))]
            g[p, pol, d] = 0.0
            if rng.random() < 0.3:
                g[p, 1 - pol, (d + 7) % 16] = 0.0
    return g


def oracle_tile_beam(oracle, sky, obs, lst, gains, res=1.28e6):
    uniq, tmap, ufreqs, fmap = oracle.unique_tile_beams(gains, obs.freqs, res)
    tabs = [oracle.tile_beam_table(sky, ty, lst, obs.latitude, uniq, ufreqs)
            if np.any(np.asarray(sky.comp_type) == ty) else None for ty in range(3)]
    return oracle.beam_struct(2, tabs, tmap, fmap, ufreqs.size), len(uniq)


@pytest.mark.parametrize("ctype", [0, 1, 2])
def test_per_tile_beams_direct_fp64(oracle, ctype):
    """Per-tile beams (each tile's own dipole gains, tiles with equal gains
    sharing one beam, evaluated at the nearest 1.28 MHz of each channel):
    the direct FP64 form against the oracle with the same explicit per-tile
    Jones table, within 1e-10."""
    pc = (0.3, math.radians(-30.0))
    obs = synth.Obs(synth.tiles_in_disk(24, 1200.0, 5), 166.4e6 + np.arange(6) * 0.64e6, pc, np.array([0.41]))
    comps = synth.point_sky(12, pc, 8.0, 3) if ctype == 0 else \
        synth.gaussians_and_shapelets(12 if ctype == 1 else 0, 0 if ctype == 1 else 8, pc, 4)
    sky = sl.SkyModelArrays.from_components(comps)
    gains = dipole_gains(obs.num_tiles, 7)
    m = SkyModeller(sky, obs.tile_xyzs, obs.freqs, pc, obs.latitude, beam="per_tile", dipole_gains=gains)
    vis = torch.zeros((obs.freqs.size, obs.num_baselines, 8), dtype=torch.float64, device="cuda")
    m.model_timestep_with(obs.lsts[0], vis)
    torch.cuda.synchronize()
    b, nuniq = oracle_tile_beam(oracle, sky, obs, obs.lsts[0], gains)
    assert nuniq > 2
    ref, _ = oracle.model_timestep(sky, obs.tile_xyzs, obs.freqs, pc, obs.lsts[0], obs.latitude, beam=b,
                                   out_f64=True)
    nrm, mx = rel_err(vis.cpu().numpy(), ref)
    assert nrm < 1e-10 and mx < 1e-10, (nrm, mx)
    # the per-tile beam is not the shared one
    vs = torch.zeros_like(vis)
    SkyModeller(sky, obs.tile_xyzs, obs.freqs, pc, obs.latitude, beam="analytic").model_timestep_with(obs.lsts[0], vs)
    torch.cuda.synchronize()
    assert rel_err(vs.cpu().numpy(), ref)[0] > 1e-4


def test_per_tile_beams_autos(oracle):
    pc = (0.3, math.radians(-30.0))
    obs = synth.Obs(synth.tiles_in_disk(16, 1200.0, 5), 166.4e6 + np.arange(4) * 0.64e6, pc, np.array([0.41]))
    sky = sl.SkyModelArrays.from_components(synth.point_sky(9, pc, 8.0, 3))
    gains = dipole_gains(obs.num_tiles, 8, damaged=0.5)
    m = SkyModeller(sky, obs.tile_xyzs, obs.freqs, pc, obs.latitude, beam="per_tile", dipole_gains=gains)
    v = torch.zeros((obs.freqs.size, obs.num_tiles, 8), dtype=torch.float32, device="cuda")
    m.model_timestep_autos_with(obs.lsts[0], v)
    torch.cuda.synchronize()
    b, _ = oracle_tile_beam(oracle, sky, obs, obs.lsts[0], gains)
    ref = oracle.model_autos(sky, obs.num_tiles, obs.freqs, obs.lsts[0], obs.latitude, beam=b)
    assert_f32_close(v.cpu().numpy(), ref, ulps=4)
