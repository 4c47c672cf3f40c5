"""libhdc's drop-in kernels beside mwa_hyperdrive's own GPU kernels
(src/gpu/model.cu, peel.cu, built for sm_100a by oracle/Makefile into
oracle/_ref/libref_gpu.so) on identical device inputs: the same FFI, the
same structs, the same buffers.

Bars: predict output (f32 visibilities) within 4 f32 ulps of the reference
kernel's; peel kernels within 1e-6 relative (f32 data); fitted ionospheric
constants within 1e-6 relative.  A larger point-source case also prints
both kernels' times (same inputs, CUDA events)."""

import ctypes
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

REF_SO = Path(__file__).resolve().parents[1] / "oracle" / "_ref" / "libref_gpu.so"
DROPIN = ["model_points", "model_gaussians", "model_shapelets", "model_autos", "xyzs_to_uvws", "rotate", "average",
          "iono_loop", "subtract_iono", "add_model"]
VEL_C = 299792458.0
LAT = synth.MWA_LAT_RAD
_KEEP = []


@pytest.fixture(scope="module")
def ref():
    if not REF_SO.exists():
        pytest.skip("reference kernels not built (oracle/Makefile needs the reference sources)")
    lib = ctypes.CDLL(str(REF_SO))
    for name in DROPIN:
        res, args = _lib.SIGNATURES[name]
        fn = getattr(lib, name)
        fn.restype, fn.argtypes = res, args
    return lib


@pytest.fixture(autouse=True)
def _release_kept():
    yield
    torch.cuda.synchronize()
    _KEEP.clear()


def dev(x, dt=np.float64):
    t = torch.from_numpy(np.ascontiguousarray(x, dt)).cuda()
    _KEEP.append(t)
    return t


def assert_f32_close(a, b, ulps=4):
    a = np.asarray(a, np.float32)
    b = np.asarray(b, np.float32)
    scale = np.maximum(np.abs(b), np.float32(np.max(np.abs(b)) * 1e-6 + 1e-30))
    bad = np.abs(a - b) > ulps * np.spacing(scale)
    assert not bad.any(), f"{bad.sum()} elements differ by more than {ulps} ulp; max diff {np.max(np.abs(a - b))}"


def rel(a, b):
    a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
    return np.linalg.norm(a - b) / np.linalg.norm(b)


def dropin_inputs(oracle, ntiles, nf, ncomp_per_group, ctype, seed, ntile_beams=3, nfreq_beams=2, want_obs=False):
    """Device inputs of the reference's model_* FFI: 3 groups (power law,
    curved power law, list) of one component type, per-tile beam Jones."""
    pc = (0.3, math.radians(-30.0))
    obs = synth.Obs(synth.tiles_in_disk(ntiles, 1500.0, seed), 160e6 + np.arange(nf) * 1.28e6, pc,
                    np.array([0.3 + 0.01]))
    rng = np.random.default_rng(seed)
    n = 3 * ncomp_per_group
    pos = synth.cap_positions(n, pc, math.radians(6.0), rng)
    comps = []
    for k in range(n):
        fd = sl.FluxDensity(150e6, float(rng.uniform(0.5, 3.0)), 0.1, -0.05, 0.02)
        g = k // ncomp_per_group
        ft = [sl.PowerLaw(-0.7, fd), sl.CurvedPowerLaw(-0.9, fd, 0.1),
              sl.FluxList([sl.FluxDensity(140e6, 2.0), sl.FluxDensity(190e6, 1.0)])][g]
        t = [sl.Point(), sl.Gaussian(2e-3, 1e-3, 0.7),
             sl.Shapelet(2e-3, 1e-3, 0.7, [sl.ShapeletCoeff(1, 0, 0.5), sl.ShapeletCoeff(2, 3, -0.2)])][ctype]
        comps.append(sl.SourceComponent(float(pos[k, 0]), float(pos[k, 1]), t, ft))
    sky = sl.SkyModelArrays.from_components(comps)
    nbl, lst = obs.num_baselines, obs.lsts[0]
    uvws = oracle.xyzs_to_cross_uvws(obs.tile_xyzs, lst - pc[0], pc[1])
    tile_map = (np.arange(ntiles) % ntile_beams).astype(np.int32)
    freq_map = (np.arange(nf) * nfreq_beams // nf).astype(np.int32)
    beam = rng.normal(size=(ntile_beams, nfreq_beams, n, 8)) * 0.3
    beam[..., 0] += 1.0
    beam[..., 6] += 1.0
    lmn = np.array([oracle.lmn_rime(c.ra, c.dec, *pc) for c in comps])
    inst150 = oracle.inst_flux(sky, [150e6])[0]
    m = ncomp_per_group
    list_fds = oracle.inst_flux(sky, obs.freqs)[:, 2 * m:3 * m]
    lm = dev(lmn).data_ptr()
    fds = dev(inst150).data_ptr()
    sis = dev(np.array([-0.7] * m + [-0.9] * m)).data_ptr()
    qs = dev(np.array([0.1] * m)).data_ptr()
    lf = dev(list_fds).data_ptr()
    gpar = dev(np.array([[2e-3, 1e-3, 0.7]] * n)).data_ptr()
    suv = oracle.shapelet_uvws(sky, obs.tile_xyzs, lst)[..., :2]  # [bl][n][2]
    suvs = [dev(suv[:, g * m:(g + 1) * m]).data_ptr() for g in range(3)]
    coeff_dt = np.dtype([("value", np.float64), ("n1", np.uint8), ("n2", np.uint8), ("pad", np.uint8, 6)])
    co = np.zeros(2 * n, coeff_dt)
    co["value"] = [0.5, -0.2] * n
    co["n1"] = [1, 2] * n
    co["n2"] = [0, 3] * n
    coeffs = dev(co.view(np.uint8), np.uint8).data_ptr()
    ncoef = dev(np.full(n, 2, np.int32), np.int32).data_ptr()
    # the reference's shapelet kernel reads the basis table through Addresses
    sbf = np.zeros(101 * 10001)
    _lib.lib().hdc_shapelet_basis(sbf.ctypes.data)
    a = _lib.Addresses(nf, nf * nbl, nbl, dev(obs.freqs).data_ptr(), dev(sbf).data_ptr(), nfreq_beams,
                       dev(tile_map, np.int32).data_ptr(), dev(freq_map, np.int32).data_ptr(),
                       dev(np.arange(ntiles, dtype=np.int32), np.int32).data_ptr())
    o = lambda g: lm + g * m * 24  # noqa: E731
    if ctype == 0:
        comps_s = _lib.Points(m, o(0), fds, sis, m, o(1), fds + m * 64, sis + m * 8, qs, m, o(2), lf)
    elif ctype == 1:
        comps_s = _lib.Gaussians(m, o(0), fds, sis, gpar, m, o(1), fds + m * 64, sis + m * 8, qs, gpar + m * 24, m,
                                 o(2), lf, gpar + 2 * m * 24)
    else:
        comps_s = _lib.Shapelets(m, o(0), fds, sis, gpar, suvs[0], coeffs, ncoef,
                                 m, o(1), fds + m * 64, sis + m * 8, qs, gpar + m * 24, suvs[1], coeffs + 2 * m * 16,
                                 ncoef + m * 4,
                                 m, o(2), lf, gpar + 2 * m * 24, suvs[2], coeffs + 4 * m * 16, ncoef + 2 * m * 4)
    if want_obs:
        return comps_s, a, dev(uvws).data_ptr(), dev(beam).data_ptr(), (nf, nbl), obs
    return comps_s, a, dev(uvws).data_ptr(), dev(beam).data_ptr(), (nf, nbl)


FN = {0: "model_points", 1: "model_gaussians", 2: "model_shapelets"}


@pytest.mark.parametrize("ctype", [0, 1, 2])
def test_f64out_variants(oracle, ref, ctype):
    """model_*_f64out: the same predict with FP64 output; rounded to FP32 it
    is the reference kernel's result (4 ulps), and it accumulates."""
    comps, a, uvws, beam, (nf, nbl) = dropin_inputs(oracle, 21, 6, 4, ctype, 31 + ctype)
    out_ref = torch.zeros((nf, nbl, 8), dtype=torch.float32, device="cuda")
    _lib.check_str(getattr(ref, FN[ctype])(ctypes.byref(comps), ctypes.byref(a), uvws, beam, out_ref.data_ptr()),
                   "reference " + FN[ctype])
    out64 = torch.zeros((nf, nbl, 8), dtype=torch.float64, device="cuda")
    fn = getattr(_lib.lib(), FN[ctype] + "_f64out")
    _lib.check_str(fn(ctypes.byref(comps), ctypes.byref(a), uvws, beam, out64.data_ptr()), FN[ctype] + "_f64out")
    torch.cuda.synchronize()
    got = out64.cpu().numpy()
    assert_f32_close(got.astype(np.float32), out_ref.cpu().numpy(), ulps=4)
    _lib.check_str(fn(ctypes.byref(comps), ctypes.byref(a), uvws, beam, out64.data_ptr()), FN[ctype] + "_f64out")
    torch.cuda.synchronize()
    np.testing.assert_allclose(out64.cpu().numpy(), 2.0 * got, rtol=1e-15, atol=0)


def test_model_points_tc(oracle):
    """model_points_tc (tensor cores, per-tile XYZs) against the FP64 predict
    of the same drop-in inputs with a beam shared by all tiles: within 1e-6
    of the rms visibility (normwise and p99.9); a per-tile beam is refused."""
    comps, a, uvws, beam, (nf, nbl), obs = dropin_inputs(oracle, 64, 5, 40, 0, 8, ntile_beams=1, nfreq_beams=2,
                                                         want_obs=True)
    ref64 = torch.zeros((nf, nbl, 8), dtype=torch.float64, device="cuda")
    _lib.check_str(_lib.lib().model_points_f64out(ctypes.byref(comps), ctypes.byref(a), uvws, beam,
                                                  ref64.data_ptr()), "model_points_f64out")
    got = torch.zeros((nf, nbl, 8), dtype=torch.float32, device="cuda")
    xyz = dev(obs.tile_xyzs)
    pc = _lib.RADec(*obs.phase_centre)
    _lib.check_str(_lib.lib().model_points_tc(ctypes.byref(comps), ctypes.byref(a), xyz.data_ptr(),
                                              float(obs.lsts[0]), pc, beam, got.data_ptr()), "model_points_tc")
    torch.cuda.synchronize()
    r = ref64.cpu().numpy()
    d = got.cpu().numpy().astype(np.float64) - r
    rms = np.sqrt(np.mean(r ** 2))
    nrm = np.sqrt(np.mean(d ** 2)) / rms
    p999 = np.quantile(np.abs(d), 0.999) / rms
    print(f"model_points_tc: normwise {nrm:.2e}, p99.9 {p999:.2e}")
    assert nrm < 1e-6 and p999 < 1e-6, (nrm, p999)


@pytest.mark.parametrize("ntiles,nbeams", [(64, 3), (97, 97), (144, 5), (256, 2), (256, 256)])
def test_model_points_tc_per_tile_beams(oracle, ntiles, nbeams):
    """model_points_tc with a beam per tile (the block form: K = 2 x
    components, operands A (B S) and A B, ten digit-plane products), any tile
    count (blocks of 128 rows x 64 columns), against the FP64 drop-in predict
    with the same per-tile beam table (itself the oracle's to 1e-10): normwise
    and p99.9 within 1e-6 of the rms visibility."""
    comps, a, uvws, beam, (nf, nbl), obs = dropin_inputs(oracle, ntiles, 4, 30, 0, ntiles + nbeams,
                                                         ntile_beams=nbeams, nfreq_beams=2, want_obs=True)
    ref64 = torch.zeros((nf, nbl, 8), dtype=torch.float64, device="cuda")
    _lib.check_str(_lib.lib().model_points_f64out(ctypes.byref(comps), ctypes.byref(a), uvws, beam,
                                                  ref64.data_ptr()), "model_points_f64out")
    got = torch.zeros((nf, nbl, 8), dtype=torch.float32, device="cuda")
    _lib.check_str(_lib.lib().model_points_tc(ctypes.byref(comps), ctypes.byref(a), dev(obs.tile_xyzs).data_ptr(),
                                              float(obs.lsts[0]), _lib.RADec(*obs.phase_centre), beam,
                                              got.data_ptr()), "model_points_tc")
    torch.cuda.synchronize()
    r = ref64.cpu().numpy()
    d = got.cpu().numpy().astype(np.float64) - r
    rms = np.sqrt(np.mean(r ** 2))
    nrm = np.sqrt(np.mean(d ** 2)) / rms
    p999 = np.quantile(np.abs(d), 0.999) / rms
    print(f"model_points_tc {ntiles} tiles, {nbeams} beams: normwise {nrm:.2e}, p99.9 {p999:.2e}")
    assert nrm < 1e-6 and p999 < 1e-6, (nrm, p999)
    # every correlation (XY and YX from the same block product) on its own
    for k in range(4):
        rk = r[..., 2 * k:2 * k + 2]
        assert np.sqrt(np.mean(d[..., 2 * k:2 * k + 2] ** 2)) < 1e-6 * np.sqrt(np.mean(rk ** 2)) * 10


@pytest.mark.parametrize("ctype", [0, 1, 2])
def test_model_kernels_match_reference_kernels(oracle, ref, ctype):
    comps, a, uvws, beam, (nf, nbl) = dropin_inputs(oracle, 21, 6, 4, ctype, 17 + ctype)
    out_ref = torch.zeros((nf, nbl, 8), dtype=torch.float32, device="cuda")
    out_hdc = torch.zeros_like(out_ref)
    _lib.check_str(getattr(ref, FN[ctype])(ctypes.byref(comps), ctypes.byref(a), uvws, beam, out_ref.data_ptr()),
                   "reference " + FN[ctype])
    _lib.check_str(getattr(_lib.lib(), FN[ctype])(ctypes.byref(comps), ctypes.byref(a), uvws, beam,
                                                   out_hdc.data_ptr()), FN[ctype])
    torch.cuda.synchronize()
    assert np.any(out_ref.cpu().numpy() != 0)
    assert_f32_close(out_hdc.cpu().numpy(), out_ref.cpu().numpy(), ulps=4)


def test_point_predict_time_beside_reference_kernel(oracle, ref):
    """128 tiles, 64 channels, 3 x 200 points, per-tile beam (1 tile beam,
    8 frequency beams): both kernels on the same inputs, CUDA events."""
    comps, a, uvws, beam, (nf, nbl) = dropin_inputs(oracle, 128, 64, 200, 0, 5, ntile_beams=1, nfreq_beams=8)
    outs = {}
    times = {}
    for name, lib in [("reference", ref), ("libhdc", _lib.lib())]:
        out = torch.zeros((nf, nbl, 8), dtype=torch.float32, device="cuda")
        fn = lib.model_points
        _lib.check_str(fn(ctypes.byref(comps), ctypes.byref(a), uvws, beam, out.data_ptr()), name)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        reps = 3
        e0.record()
        for _ in range(reps):
            _lib.check_str(fn(ctypes.byref(comps), ctypes.byref(a), uvws, beam, out.data_ptr()), name)
        e1.record()
        torch.cuda.synchronize()
        times[name] = e0.elapsed_time(e1) / reps
        out.zero_()
        _lib.check_str(fn(ctypes.byref(comps), ctypes.byref(a), uvws, beam, out.data_ptr()), name)
        torch.cuda.synchronize()
        outs[name] = out.cpu().numpy()
    work = nbl * nf * 600
    print(f"model_points 128 tiles x 64 ch x 600 points: reference {times['reference']:.2f} ms "
          f"({work / times['reference'] / 1e6:.3g} Gvis.comp/s), libhdc {times['libhdc']:.2f} ms "
          f"({work / times['libhdc'] / 1e6:.3g} Gvis.comp/s), ratio {times['reference'] / times['libhdc']:.2f}")
    assert_f32_close(outs["libhdc"], outs["reference"], ulps=4)


def peel_setup(seed=0, ntiles=16, nt=2, nf=8):
    rng = np.random.default_rng(seed)
    pc = (0.1, math.radians(-27.0))
    xyzs = synth.tiles_in_disk(ntiles, 1500.0, seed + 1)
    freqs = 165e6 + np.arange(nf) * 1.28e6
    lmsts = pc[0] + np.arange(nt) * 8.0 * synth.SIDEREAL_RATE
    return rng, pc, xyzs, freqs, lmsts


def test_peel_kernels_match_reference_kernels(ref):
    rng, pc, xyzs, freqs, lmsts = peel_setup()
    nt, nf, ntiles = lmsts.size, freqs.size, xyzs.shape[0]
    nbl = ntiles * (ntiles - 1) // 2
    lam = VEL_C / freqs
    xyz_t = np.broadcast_to(xyzs, (nt, ntiles, 3)).copy()
    src = (0.13, math.radians(-25.0))
    ours = _lib.lib()
    uv = {}
    for name, lib in [("ref", ref), ("hdc", ours)]:
        u = torch.zeros((nt, nbl, 3), dtype=torch.float64, device="cuda")
        _lib.check_str(lib.xyzs_to_uvws(dev(xyz_t).data_ptr(), dev(lmsts).data_ptr(), u.data_ptr(), _lib.RADec(*src),
                                        ntiles, nbl, nt), name)
        uv[name] = u
    torch.cuda.synchronize()
    np.testing.assert_allclose(uv["hdc"].cpu().numpy(), uv["ref"].cpu().numpy(), rtol=0, atol=1e-9)
    frm = torch.zeros_like(uv["ref"])
    _lib.check_str(ref.xyzs_to_uvws(dev(xyz_t).data_ptr(), dev(lmsts).data_ptr(), frm.data_ptr(), _lib.RADec(*pc),
                                    ntiles, nbl, nt), "ref")
    vis = rng.normal(size=(nt, nf, nbl, 8)).astype(np.float32)
    w = rng.uniform(0.0, 2.0, (nt, nf, nbl)).astype(np.float32)
    w[:, :, ::7] = 0.0
    model = rng.normal(size=(nt, nf, nbl, 8)).astype(np.float32)
    c, old = (1.3e-5, -2.1e-5, 1.04), (0.4e-5, 0.9e-5, 0.97)
    res = {}
    for name, lib in [("ref", ref), ("hdc", ours)]:
        v = dev(vis, np.float32)
        _lib.check_str(lib.rotate(v.data_ptr(), nt, nbl, nf, frm.data_ptr(), uv["ref"].data_ptr(),
                                  dev(lam).data_ptr()), name)
        lo = torch.zeros((nf // 4, nbl, 8), dtype=torch.float32, device="cuda")
        _lib.check_str(lib.average(dev(vis, np.float32).data_ptr(), dev(w, np.float32).data_ptr(), lo.data_ptr(), nt,
                                   nbl, nf, 4), name)
        am = dev(vis, np.float32)
        _lib.check_str(lib.add_model(am.data_ptr(), dev(model, np.float32).data_ptr(), _lib.IonoConsts(*c),
                                     dev(lam).data_ptr(), uv["ref"].data_ptr(), nt, nf, nbl), name)
        si = dev(vis, np.float32)
        _lib.check_str(lib.subtract_iono(si.data_ptr(), dev(model, np.float32).data_ptr(), _lib.IonoConsts(*c),
                                         _lib.IonoConsts(*old), uv["ref"].data_ptr(), dev(lam).data_ptr(), nt, nbl,
                                         nf), name)
        torch.cuda.synchronize()
        res[name] = [x.cpu().numpy() for x in (v, lo, am, si)]
    for k, what in enumerate(["rotate", "average", "add_model", "subtract_iono"]):
        assert rel(res["hdc"][k], res["ref"][k]) < 1e-6, what


def test_iono_loop_matches_reference_kernel(ref):
    rng, pc, xyzs, freqs, lmsts = peel_setup(ntiles=24, nf=12)
    ntiles = xyzs.shape[0]
    nbl = ntiles * (ntiles - 1) // 2
    lam = VEL_C / freqs
    uvw = np.zeros((nbl, 3))
    i, j = np.triu_indices(ntiles, 1)
    uvw[:, :2] = (xyzs[i, :2] - xyzs[j, :2])
    model = np.zeros((freqs.size, nbl, 8), np.float32)
    amp = rng.lognormal(0, 0.3, (freqs.size, nbl))
    model[..., 0] = amp
    model[..., 6] = amp
    a, b, g = 2e-5, -1.5e-5, 1.05
    ph = np.exp(1j * (-2 * np.pi * (uvw[:, 0] * a + uvw[:, 1] * b))[None, :] * lam[:, None]) * g
    v = (model[..., 0::2] + 1j * model[..., 1::2]) * ph[..., None]
    resid = np.empty_like(model)
    resid[..., 0::2], resid[..., 1::2] = v.real, v.imag
    w = np.ones((freqs.size, nbl), np.float32)
    consts = {}
    for name, lib in [("ref", ref), ("hdc", _lib.lib())]:
        c = _lib.IonoConsts(0.0, 0.0, 1.0)
        rot = torch.zeros((freqs.size, nbl, 8), dtype=torch.float32, device="cuda")
        fits = torch.zeros((freqs.size, nbl, 8), dtype=torch.float64, device="cuda")
        _lib.check_str(lib.iono_loop(dev(resid, np.float32).data_ptr(), dev(w, np.float32).data_ptr(),
                                     dev(model, np.float32).data_ptr(), rot.data_ptr(), fits.data_ptr(),
                                     ctypes.byref(c), nbl, freqs.size, 10, dev(uvw).data_ptr(), dev(lam).data_ptr(),
                                     1.0), name)
        torch.cuda.synchronize()
        consts[name] = (c.alpha, c.beta, c.gain)
    for x, y in zip(consts["hdc"], consts["ref"]):
        assert abs(x - y) <= 1e-6 * abs(y), (consts["hdc"], consts["ref"])
