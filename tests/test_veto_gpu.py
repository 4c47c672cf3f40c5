"""The source-list veto: the GPU brightness (hdc_source_brightness) against
the CPU oracle's flux and beam restatements, the reference's no-beam
known answer, and veto_sources' drop / threshold / sort / top-N rules
(srclist/veto.rs:44-188)."""

import math

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("no CUDA device", allow_module_level=True)

from mwa_hyperdrive_b200 import srclist as sl  # noqa: E402
from mwa_hyperdrive_b200 import srclist_io as io  # noqa: E402
from mwa_hyperdrive_b200 import synth  # noqa: E402

LAT = synth.MWA_LAT_RAD


def point(ra_deg, dec_deg, i, si=-0.8, freq=180e6):
    return sl.SourceComponent(math.radians(ra_deg), math.radians(dec_deg), sl.Point(),
                              sl.PowerLaw(si, sl.FluxDensity(freq, i)))


def test_no_beam_known_answer():
    """veto.rs:224-246: 1 Jy of Stokes I gives a beam-attenuated flux of 2
    with no beam, at the zenith as anywhere."""
    lst = 0.3
    s = sl.SourceList()
    s["zenith"] = sl.Source([point(math.degrees(lst), math.degrees(LAT), 1.0, si=0.0)])
    s["low"] = sl.Source([point(math.degrees(lst) + 60.0, math.degrees(LAT) - 50.0, 1.0, si=0.0)])
    out = io.veto_sources(s, (lst, LAT), lst, LAT, [180e6], beam="none", veto_threshold=0.0)
    assert list(out.keys()) == ["zenith", "low"] or list(out.keys()) == ["low", "zenith"]
    b = brightness(s, (lst, LAT), lst, [180e6], "none")
    np.testing.assert_allclose(b, [2.0, 2.0], rtol=1e-15)


def brightness(s, pc, lst, freqs, beam, cutoff_deg=180.0, min_el_deg=0.0):
    import ctypes

    from mwa_hyperdrive_b200 import _lib

    names = list(s.keys())
    comps, owner = [], []
    for k, n in enumerate(names):
        for c in s[n].components:
            comps.append(c)
            owner.append(k)
    sky = sl.SkyModelArrays.from_components(comps)
    owner = np.ascontiguousarray(owner, np.int32)
    fr = np.ascontiguousarray(freqs, np.float64)
    out = np.zeros(len(names))
    _lib.check(_lib.lib().hdc_source_brightness(ctypes.byref(sky.struct()), owner.ctypes.data, len(names),
                                                fr.ctypes.data, fr.size, lst, LAT, _lib.RADec(*pc),
                                                {"none": 0, "analytic": 1}[beam], math.radians(cutoff_deg),
                                                math.radians(min_el_deg), out.ctypes.data), "brightness")
    return out


def test_brightness_matches_oracle(oracle):
    """Per source: the smallest over the coarse frequencies of the summed
    |XX| + |YY| of J I J^H, with the oracle's flux estimate and beam."""
    rng = np.random.default_rng(5)
    pc = (0.2, math.radians(-27.0))
    lst = 0.25
    s = sl.SourceList()
    for k in range(40):
        comps = []
        for _ in range(int(rng.integers(1, 4))):
            ra = (math.degrees(pc[0]) + rng.uniform(-30, 30)) % 360.0
            dec = math.degrees(pc[1]) + rng.uniform(-30, 30)
            fd = sl.FluxDensity(150e6, float(rng.lognormal()), float(rng.normal() * 0.05), float(rng.normal() * 0.05),
                                float(rng.normal() * 0.02))
            ft = [sl.PowerLaw(-0.8, fd), sl.CurvedPowerLaw(-0.7, fd, 0.1),
                  sl.FluxList([fd, sl.FluxDensity(200e6, fd.i * 0.7)])][k % 3]
            comps.append(sl.SourceComponent(math.radians(ra), math.radians(dec), sl.Point(), ft))
        s[f"s{k}"] = sl.Source(comps)
    freqs = [167.68e6, 182.4e6, 197.12e6]
    for beam in ("none", "analytic"):
        got = brightness(s, pc, lst, freqs, beam)
        exp = []
        for n in s:
            sky = sl.SkyModelArrays.from_components(s[n].components)
            inst = oracle.inst_flux(sky, freqs)  # [f][c][8]
            tot = np.zeros(len(freqs))
            for c, comp in enumerate(s[n].components):
                az, el = oracle.hadec_to_azel(lst - comp.ra, comp.dec, LAT)
                for f, nu in enumerate(freqs):
                    i = inst[f, c]
                    I = np.array([[i[0] + 1j * i[1], i[2] + 1j * i[3]], [i[4] + 1j * i[5], i[6] + 1j * i[7]]])
                    if beam == "analytic":
                        b = oracle.analytic_beam(az, el, nu)
                        J = np.array([[b[0] + 1j * b[1], b[2] + 1j * b[3]], [b[4] + 1j * b[5], b[6] + 1j * b[7]]])
                        I = J @ I @ J.conj().T
                    tot[f] += abs(I[0, 0]) + abs(I[1, 1])
            exp.append(tot.min())
        np.testing.assert_allclose(got, exp, rtol=1e-12)


def test_veto_rules():
    """Drops: a component below the horizon, one outside the distance cutoff,
    a source below the threshold; the rest brightest first, top N, and an
    error when fewer than N survive."""
    lst, pc = 0.0, (0.0, math.radians(-27.0))
    s = sl.SourceList()
    s["dim"] = sl.Source([point(1.0, -27.0, 0.001)])
    s["bright"] = sl.Source([point(359.0, -26.0, 10.0)])
    s["medium"] = sl.Source([point(2.0, -30.0, 1.0), point(3.0, -31.0, 1.5)])
    s["below_horizon"] = sl.Source([point(2.0, -30.0, 50.0), point(180.0, 60.0, 1.0)])
    s["far"] = sl.Source([point(60.0, -27.0, 30.0)])
    s["faint"] = sl.Source([point(5.0, -20.0, 0.5)])
    out = io.veto_sources(s, pc, lst, LAT, [167.68e6, 197.12e6], beam="none", source_dist_cutoff_deg=40.0,
                          veto_threshold=0.1)
    assert list(out.keys()) == ["bright", "medium", "faint"]
    top = io.veto_sources(s, pc, lst, LAT, [167.68e6, 197.12e6], beam="none", num_sources=2,
                          source_dist_cutoff_deg=40.0, veto_threshold=0.1)
    assert list(top.keys()) == ["bright", "medium"]
    with pytest.raises(io.SourceListError):
        io.veto_sources(s, pc, lst, LAT, [167.68e6], beam="none", num_sources=5, source_dist_cutoff_deg=40.0,
                        veto_threshold=0.1)
    # the analytic beam attenuates away from the zenith: the order can change
    # but the veto still drops the same sources
    outb = io.veto_sources(s, pc, lst, LAT, [167.68e6, 197.12e6], beam="analytic", source_dist_cutoff_deg=40.0,
                           veto_threshold=0.01)
    assert set(outb.keys()) == {"bright", "medium", "faint"}
