"""The FEE beam on the GPU (csrc/fee.cu through the C ABI) against the CPU
oracle (oracle/fee_ref.py), and the modeller's predict with an FEE beam per
tile against the oracle predict given the oracle's FEE Jones tables.

Tolerances: the Jones matrices within 1e-12 of the largest element (FP64,
different summation orders); the FP64 predict within 1e-10 (normwise and
per visibility over the rms), the tensor form within 1e-6.  Parity with
mwa_hyperbeam itself is unpinned (no hyperbeam, no beam file here); the
coefficients are seeded synthetic ones with the file's layout.
"""

import ctypes
import math

import numpy as np
import pytest

from mwa_hyperdrive_b200 import srclist as sl
from mwa_hyperdrive_b200 import synth
from oracle import fee_ref as fr

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("no CUDA device", allow_module_level=True)

from mwa_hyperdrive_b200 import _lib  # noqa: E402
from mwa_hyperdrive_b200.fee import FeeBeam  # noqa: E402
from mwa_hyperdrive_b200.model import SkyModeller  # noqa: E402

LAT = synth.MWA_LAT_RAD
FILE = synth.fee_coeffs([166400000, 167680000, 168960000, 170240000], [8, 9, 10, 9], seed=5)


def tile_settings(ntiles, seed):
    """Delays [tile][16] and gains [tile][32]: a pointing shared by most
    tiles, a few tiles with a dead dipole (delay 32) or a low gain, so that
    tiles share beams."""
    rng = np.random.default_rng(seed)
    base = np.array([(d % 4) * 2 + (d // 4) for d in range(16)], np.uint32)
    delays = np.tile(base, (ntiles, 1))
    amps = np.ones((ntiles, 32))
    for t in range(ntiles):
        r = rng.random()
        if r < 0.2:
            delays[t, rng.integers(16)] = 32
        elif r < 0.35:
            amps[t, rng.integers(32)] = 0.5
    return delays, amps


def oracle_tables(file, az, za, freqs, delays, amps, tmap, fmap, norm=True, lat=None):
    """[uniq tile][uniq freq][dir][8] in the library's unique order."""
    nu, nuf = int(tmap.max()) + 1, int(fmap.max()) + 1
    out = np.zeros((nu, nuf, np.size(az), 8))
    for u in range(nu):
        t = int(np.argmax(tmap == u))
        for uf in range(nuf):
            f = int(np.argmax(fmap == uf))
            j = fr.calc_jones(file, az, za, freqs[f], delays[t], amps[t], norm_to_zenith=norm, latitude=lat)
            out[u, uf] = fr.as_jones8(j)
    return out


@pytest.mark.parametrize("norm,lat", [(True, LAT), (True, None), (False, None)])
def test_calc_jones_against_the_oracle(norm, lat):
    rng = np.random.default_rng(2)
    n = 150
    az = rng.uniform(0.0, 2 * math.pi, n)
    za = rng.uniform(0.0, 1.55, n)
    # the zenith and the horizon; with the rotation, directions next to the
    # zenith (there the parallactic angle is atan2 of two rounding-level
    # numbers, undefined at the zenith itself)
    az[:3], za[:3] = [0.0, 1.0, 4.0], [0.0 if lat is None else 1e-3, 0.0 if lat is None else 2e-3, math.pi / 2]
    freqs = 166.4e6 + np.arange(12) * 0.32e6  # channels over all four file frequencies
    delays, amps = tile_settings(20, 3)
    beam = FeeBeam(FILE, freqs, delays, amps, norm_to_zenith=norm)
    tmap, fmap = beam.maps()
    assert 2 < beam.num_unique_tiles() < 20 and beam.num_unique_freqs() == 4
    got = beam.calc_jones(az, za, latitude_rad=lat).cpu().numpy()
    torch.cuda.synchronize()
    ref = oracle_tables(FILE, az, za, freqs, delays, amps, tmap, fmap, norm, lat)
    err = np.max(np.abs(got - ref)) / np.max(np.abs(ref))
    assert err < 1e-12, err


def test_maps_and_gains_forms():
    """Tiles with the same delays and gains share a beam, a dead dipole is a
    zero gain, 16 gains serve both polarisations, and each channel maps to its
    closest file frequency."""
    freqs = np.array([166.0e6, 166.41e6, 167.1e6, 168.2e6, 171.0e6, 167.04e6])
    delays = np.zeros((5, 16), np.uint32)
    delays[2, 7] = 32
    amps = np.ones((5, 16))
    amps[3, 2] = 0.0
    beam = FeeBeam(FILE, freqs, delays, amps)
    tmap, fmap = beam.maps()
    assert list(tmap) == [0, 0, 1, 2, 0]
    file_f = FILE["freqs_hz"].astype(np.int64)
    closest = [int(np.argmin(np.abs(file_f - int(round(f))))) for f in freqs]
    order = list(dict.fromkeys(closest))
    assert list(fmap) == [order.index(c) for c in closest]
    az, za = np.array([0.5, 2.5]), np.array([0.4, 1.0])
    got = beam.calc_jones(az, za, latitude_rad=LAT).cpu().numpy()
    a32 = np.ones((5, 32))
    a32[2, 7] = a32[2, 23] = 0.0
    a32[3, 2] = a32[3, 18] = 0.0
    ref = oracle_tables(FILE, az, za, freqs, np.where(delays == 32, 0, delays), a32, tmap, fmap, True, LAT)
    assert np.max(np.abs(got - ref)) / np.max(np.abs(ref)) < 1e-12


def test_argument_errors():
    lib = _lib.lib()
    freqs = np.array([167.68e6])
    delays = np.zeros((2, 16), np.uint32)
    amps = np.ones((2, 32))
    with pytest.raises(_lib.HdcError):
        FeeBeam(FILE, freqs, np.full((2, 16), 33, np.uint32), amps)  # delays above 32
    beam = FeeBeam(FILE, freqs, delays, amps)
    out = torch.empty(8, dtype=torch.float64, device="cuda")
    d = torch.zeros(1, dtype=torch.float64, device="cuda")
    assert lib.hdc_fee_calc_jones(beam.handle, d.data_ptr(), d.data_ptr(), 1, None, 1, out.data_ptr(), None) == 5
    # a modeller with another tile count refuses the beam
    sky = sl.SkyModelArrays.from_components(synth.point_sky(3, (0.0, -0.47), 5.0, 1))
    m = SkyModeller(sky, synth.tiles_in_disk(3, 500.0, 1), freqs, (0.0, -0.47), LAT)
    with pytest.raises(_lib.HdcError):
        m.set_fee_beam(beam)


def comp_azza(oracle, sky, ctype, lst, lat):
    sel = np.asarray(sky.comp_type) == ctype
    az, za = [], []
    for ra, dec in zip(sky.ra[sel], sky.dec[sel]):
        a, e = oracle.hadec_to_azel(lst - ra, dec, lat)
        az.append(a)
        za.append(math.pi / 2 - e)
    return np.array(az), np.array(za)


@pytest.mark.parametrize("ctype", [0, 1, 2])
def test_modeller_with_fee_beam_fp64(oracle, ctype):
    """The direct FP64 predict with an FEE beam per tile, evaluated on the
    device per timestep, against the oracle predict given the oracle's FEE
    Jones of every component, within 1e-10."""
    pc = (0.3, math.radians(-30.0))
    obs = synth.Obs(synth.tiles_in_disk(18, 1200.0, 5), 166.4e6 + np.arange(6) * 0.64e6, pc, np.array([0.41]))
    comps = synth.point_sky(10, pc, 8.0, 3) if ctype == 0 else \
        synth.gaussians_and_shapelets(10 if ctype == 1 else 0, 0 if ctype == 1 else 6, pc, 4)
    sky = sl.SkyModelArrays.from_components(comps)
    delays, amps = tile_settings(obs.num_tiles, 9)
    beam = FeeBeam(FILE, obs.freqs, delays, amps)
    tmap, fmap = beam.maps()
    m = SkyModeller(sky, obs.tile_xyzs, obs.freqs, pc, obs.latitude, beam="fee", fee_beam=beam)
    vis = torch.zeros((obs.freqs.size, obs.num_baselines, 8), dtype=torch.float64, device="cuda")
    m.model_timestep_with(obs.lsts[0], vis)
    torch.cuda.synchronize()
    az, za = comp_azza(oracle, sky, ctype, obs.lsts[0], obs.latitude)
    tab = oracle_tables(FILE, az, za, obs.freqs, delays, amps, tmap, fmap, True, obs.latitude)
    tabs = [tab if t == ctype else None for t in range(3)]
    b = oracle.beam_struct(2, tabs, tmap, fmap, beam.num_unique_freqs())
    ref, _ = oracle.model_timestep(sky, obs.tile_xyzs, obs.freqs, pc, obs.lsts[0], obs.latitude, beam=b,
                                   out_f64=True)
    got = vis.cpu().numpy()
    nrm = np.linalg.norm(got - ref) / np.linalg.norm(ref)
    mx = np.max(np.abs(got - ref)) / (np.linalg.norm(ref) / math.sqrt(ref.size))
    assert nrm < 1e-10 and mx < 1e-10, (nrm, mx)


def test_modeller_with_fee_beam_tensor_form(oracle):
    """The chosen form with the FEE beam per tile -- the tensor-core points
    (block form), the FP32 per-tile Gaussians and shapelets -- against the
    same oracle, within 1e-6."""
    pc = (0.3, math.radians(-30.0))
    obs = synth.Obs(synth.tiles_in_disk(40, 1500.0, 6), 166.4e6 + np.arange(4) * 0.64e6, pc, np.array([0.37]))
    sky = sl.SkyModelArrays.from_components(synth.point_sky(64, pc, 8.0, 7) +
                                            synth.gaussians_and_shapelets(20, 6, pc, 5))
    delays, amps = tile_settings(obs.num_tiles, 10)
    beam = FeeBeam(FILE, obs.freqs, delays, amps)
    tmap, fmap = beam.maps()
    m = SkyModeller(sky, obs.tile_xyzs, obs.freqs, pc, obs.latitude, beam="fee", fee_beam=beam, form="tensor")
    vis = torch.zeros((obs.freqs.size, obs.num_baselines, 8), dtype=torch.float64, device="cuda")
    m.model_timestep_with(obs.lsts[0], vis)
    torch.cuda.synchronize()
    tabs = []
    for ty in range(3):
        az, za = comp_azza(oracle, sky, ty, obs.lsts[0], obs.latitude)
        tabs.append(oracle_tables(FILE, az, za, obs.freqs, delays, amps, tmap, fmap, True, obs.latitude))
    b = oracle.beam_struct(2, tabs, tmap, fmap, beam.num_unique_freqs())
    ref, _ = oracle.model_timestep(sky, obs.tile_xyzs, obs.freqs, pc, obs.lsts[0], obs.latitude, beam=b,
                                   out_f64=True)
    got = vis.cpu().numpy()
    nrm = np.linalg.norm(got - ref) / np.linalg.norm(ref)
    assert nrm < 1e-6, nrm


def test_veto_brightness_with_the_fee_beam(oracle):
    """hdc_source_brightness_fee (veto_sources with the FEE beam: no tile, so
    the ideal delays and unit gains) against the oracle's flux estimates and
    FEE Jones, and veto_sources' beam="fee" path."""
    from mwa_hyperdrive_b200 import srclist_io as io

    rng = np.random.default_rng(8)
    pc = (0.2, math.radians(-27.0))
    lst = 0.25
    s = sl.SourceList()
    for k in range(25):
        comps = []
        for _ in range(int(rng.integers(1, 4))):
            ra = (math.degrees(pc[0]) + rng.uniform(-25, 25)) % 360.0
            dec = math.degrees(pc[1]) + rng.uniform(-25, 25)
            fd = sl.FluxDensity(150e6, float(rng.lognormal()), 0.0, 0.0, 0.0)
            comps.append(sl.SourceComponent(math.radians(ra), math.radians(dec), sl.Point(), sl.PowerLaw(-0.8, fd)))
        s[f"s{k}"] = sl.Source(comps)
    freqs = np.array([166.4e6, 168.96e6, 170.24e6])
    ideal = np.array([(d % 4) + (d // 4) for d in range(16)], np.uint32)
    beam = FeeBeam(FILE, freqs, ideal[None, :], np.ones((1, 32)))
    names = list(s.keys())
    comps, owner = [], []
    for k, n in enumerate(names):
        for c in s[n].components:
            comps.append(c)
            owner.append(k)
    sky = sl.SkyModelArrays.from_components(comps)
    owner = np.ascontiguousarray(owner, np.int32)
    got = np.zeros(len(names))
    _lib.check(_lib.lib().hdc_source_brightness_fee(ctypes.byref(sky.struct()), owner.ctypes.data, len(names),
                                                    freqs.ctypes.data, freqs.size, lst, LAT, _lib.RADec(*pc),
                                                    beam.handle, math.radians(180.0), 0.0, got.ctypes.data),
               "hdc_source_brightness_fee")
    exp = np.zeros(len(names))
    inst = oracle.inst_flux(sky, freqs)  # [f][c][8]
    tot = np.zeros((len(names), freqs.size))
    for c, comp in enumerate(comps):
        az, el = oracle.hadec_to_azel(lst - comp.ra, comp.dec, LAT)
        for f, nu in enumerate(freqs):
            j = fr.calc_jones(FILE, az, math.pi / 2 - el, nu, ideal, np.ones(32), latitude=LAT)[0]
            J = j.reshape(2, 2)
            i = inst[f, c]
            inst_j = np.array([[i[0] + 1j * i[1], i[2] + 1j * i[3]], [i[4] + 1j * i[5], i[6] + 1j * i[7]]])
            m = J @ inst_j @ J.conj().T
            tot[owner[c], f] += abs(m[0, 0]) + abs(m[1, 1])
    below = np.array([any(oracle.hadec_to_azel(lst - c.ra, c.dec, LAT)[1] < 0.0 for c in s[n].components)
                      for n in names])
    exp = np.where(below, -1.0, tot.min(axis=1))
    np.testing.assert_allclose(got, exp, rtol=1e-11)
    out = io.veto_sources(s, pc, lst, LAT, freqs, beam="fee", fee_beam=beam, veto_threshold=0.05)
    keep = sorted([(exp[k], n) for k, n in enumerate(names) if exp[k] >= 0.05], key=lambda t: -t[0])
    assert list(out.keys()) == [n for _, n in keep]
    with pytest.raises(_lib.HdcError):  # a beam of two tiles is not the reference's tile-less beam
        two = FeeBeam(FILE, freqs, np.stack([ideal, ideal + 1]), np.ones((2, 32)))
        io.veto_sources(s, pc, lst, LAT, freqs, beam="fee", fee_beam=two)


def test_autos_with_fee_beam(oracle):
    """model_timestep_autos_with with the FEE beam per tile against the
    oracle's autos given the oracle's FEE tables (f32 output within 4 ulps of
    the oracle's identically demoted result)."""
    pc = (0.3, math.radians(-30.0))
    obs = synth.Obs(synth.tiles_in_disk(12, 1000.0, 4), 166.4e6 + np.arange(4) * 0.64e6, pc, np.array([0.41]))
    sky = sl.SkyModelArrays.from_components(synth.point_sky(8, pc, 8.0, 3) +
                                            synth.gaussians_and_shapelets(4, 2, pc, 6))
    delays, amps = tile_settings(obs.num_tiles, 12)
    beam = FeeBeam(FILE, obs.freqs, delays, amps)
    tmap, fmap = beam.maps()
    m = SkyModeller(sky, obs.tile_xyzs, obs.freqs, pc, obs.latitude, beam="fee", fee_beam=beam)
    v = torch.zeros((obs.freqs.size, obs.num_tiles, 8), dtype=torch.float32, device="cuda")
    m.model_timestep_autos_with(obs.lsts[0], v)
    torch.cuda.synchronize()
    tabs = []
    for ty in range(3):
        az, za = comp_azza(oracle, sky, ty, obs.lsts[0], obs.latitude)
        tabs.append(oracle_tables(FILE, az, za, obs.freqs, delays, amps, tmap, fmap, True, obs.latitude))
    b = oracle.beam_struct(2, tabs, tmap, fmap, beam.num_unique_freqs())
    ref = oracle.model_autos(sky, obs.num_tiles, obs.freqs, obs.lsts[0], obs.latitude, beam=b)
    got = v.cpu().numpy().astype(np.float32)
    ref = np.asarray(ref, np.float32)
    scale = np.maximum(np.abs(ref), np.float32(np.max(np.abs(ref)) * 1e-6 + 1e-30))
    assert not (np.abs(got - ref) > 4 * np.spacing(scale)).any(), np.max(np.abs(got - ref))


def test_calc_jones_at_degree_30(oracle):
    """Degrees up to 30, where the recurrences' dynamic range is largest
    ((2m - 1)!! against the small C_mn): within 1e-8 of the largest element.
    The bar is the oracle's own: its Legendre series (numpy's) agrees with
    scipy's lpmv to 1.5e-9 of a column's largest value at degree 40 and
    loses digits with degree."""
    file = synth.fee_coeffs([167680000, 168960000], [28, 30], seed=9)
    rng = np.random.default_rng(4)
    n = 64
    az = rng.uniform(0.0, 2 * math.pi, n)
    za = rng.uniform(0.0, 1.5, n)
    freqs = np.array([167.68e6, 168.96e6])
    delays = np.stack([np.arange(16, dtype=np.uint32) % 5, np.full(16, 3, np.uint32)])
    delays[1, 6] = 32
    amps = np.ones((2, 32))
    beam = FeeBeam(file, freqs, delays, amps)
    tmap, fmap = beam.maps()
    got = beam.calc_jones(az, za, latitude_rad=LAT).cpu().numpy()
    torch.cuda.synchronize()
    ref = oracle_tables(file, az, za, freqs, delays, amps, tmap, fmap, True, LAT)
    err = np.max(np.abs(got - ref)) / np.max(np.abs(ref))
    assert err < 1e-8, err


def test_zero_zenith_norm_is_refused():
    """A coefficient set whose zenith-pointed beam has a zero element at the
    zenith cannot be normalised to it: hdc_fee_beam_new refuses it (and the
    same set without normalisation is accepted)."""
    file = synth.fee_coeffs([167680000], 4, seed=2)
    file["q"] = file["q"].copy()
    file["q"][0, 0] = 0.0  # no X coefficients at all
    delays = np.zeros((1, 16), np.uint32)
    with pytest.raises(_lib.HdcError, match="cannot normalise"):
        FeeBeam(file, [167.68e6], delays, np.ones((1, 32)), norm_to_zenith=True)
    FeeBeam(file, [167.68e6], delays, np.ones((1, 32)), norm_to_zenith=False).close()
