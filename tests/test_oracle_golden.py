"""Pin the CPU oracle against mwa_hyperdrive's own known-answer tests.

Predictor KATs come from src/model/tests/{mod,cpu}.rs (no-beam cases, which
the reference checks with epsilon = 0); DI-calibration KATs restate
src/di_calibrate/tests.rs; the shapelet basis table is checked against the
reference generator's values and src/model/shapelets.rs:44-59.
"""

import json
import math
from pathlib import Path

import numpy as np
import pytest

from mwa_hyperdrive_b200 import srclist as sl
from mwa_hyperdrive_b200 import synth

GOLD = Path(__file__).resolve().parent / "golden"
KATS = json.loads((GOLD / "model_kats.json").read_text())
MWA_LAT_RAD = -0.4660608448386394  # marlu MWA_LAT_RAD (-26.703319 deg)


def obs():
    o = KATS["obs"]
    pc = tuple(math.radians(x) for x in o["phase_centre_deg"])
    return pc, np.array(o["freqs_hz"]), o["lst_rad"], np.array(o["xyzs"], dtype=np.float64)


def flux(kind):
    # src/model/tests/mod.rs:125-166
    if kind == "list":
        return sl.FluxList([sl.FluxDensity(150e6, 1.0), sl.FluxDensity(175e6, 3.0), sl.FluxDensity(200e6, 2.0)])
    if kind == "power_law":
        return sl.PowerLaw(-0.8, sl.FluxDensity(150e6, 1.0))
    return sl.CurvedPowerLaw(-0.8, sl.FluxDensity(150e6, 1.0), 0.03)


def comp(kind, pos_deg, ctype):
    ra, dec = sl.radec_deg(*pos_deg)
    if ctype == 0:
        t = sl.Point()
    elif ctype == 1:
        t = sl.Gaussian(0.0, 0.0, 0.0)
    else:
        t = sl.Shapelet(0.0, 0.0, 0.0, [sl.ShapeletCoeff(0, 0, 1.0)])
    return sl.SourceComponent(ra, dec, t, flux(kind))


def golden(name):
    g = np.array(KATS["cases"][name], dtype=np.float32)  # [f][bl][4][2]
    return g.reshape(3, 3, 8)


CASES = [
    ("list", (0.0, -27.0), "test_list_zenith_visibilities"),
    ("power_law", (0.0, -27.0), "test_power_law_zenith_visibilities"),
    ("curved_power_law", (0.0, -27.0), "test_curved_power_law_zenith_visibilities"),
    ("list", (1.0, -27.0), "test_list_off_zenith_visibilities"),
    ("power_law", (1.0, -27.0), "test_power_law_off_zenith_visibilities"),
    ("curved_power_law", (1.0, -27.0), "test_curved_power_law_off_zenith_visibilities"),
]


@pytest.mark.parametrize("ctype", [0, 1, 2])
@pytest.mark.parametrize("kind,pos,name", CASES)
def test_predictor_kats_exact(oracle, ctype, kind, pos, name):
    pc, freqs, lst, xyzs = obs()
    sky = sl.SkyModelArrays.from_components([comp(kind, pos, ctype)])
    uvws = oracle.xyzs_to_cross_uvws(xyzs, lst - pc[0], pc[1])
    vis = oracle.model_type(ctype, sky, xyzs, freqs, pc, lst, MWA_LAT_RAD, uvws)
    # The reference asserts epsilon = 0 for the no-beam cases.
    np.testing.assert_array_equal(vis, golden(name))


@pytest.mark.parametrize("ctype,name", [(1, "test_multiple_gaussian_components"),
                                        (2, "test_multiple_shapelet_components")])
def test_multiple_components_exact(oracle, ctype, name):
    pc, freqs, lst, xyzs = obs()
    sky = sl.SkyModelArrays.from_components([comp("list", (1.0, -27.0), ctype), comp("list", (1.1, -27.0), ctype)])
    uvws = oracle.xyzs_to_cross_uvws(xyzs, lst - pc[0], pc[1])
    vis = oracle.model_type(ctype, sky, xyzs, freqs, pc, lst, MWA_LAT_RAD, uvws)
    np.testing.assert_array_equal(vis, golden(name))


def test_shapelet_uvws_exact(oracle):
    pc, freqs, lst, xyzs = obs()
    sky = sl.SkyModelArrays.from_components([comp("list", (1.0, -27.0), 2), comp("list", (1.1, -27.0), 2)])
    suv = oracle.shapelet_uvws(sky, xyzs, 0.0)
    suv[..., 2] = 0.0
    np.testing.assert_array_equal(suv, np.array(KATS["shapelet_uvws_bl_comp"]))


def test_model_timestep_and_autos(oracle):
    # model/tests/cpu.rs:332-367 (precession off) and 440-576 (autos)
    pc, freqs, lst, xyzs = obs()
    sky = sl.SkyModelArrays.from_components([comp("list", (0.0, -27.0), 0)])
    vis, uvws = oracle.model_timestep(sky, xyzs, freqs, pc, lst, MWA_LAT_RAD)
    np.testing.assert_array_equal(vis, golden("test_list_zenith_visibilities"))
    autos = oracle.model_autos(sky, 3, freqs, lst, MWA_LAT_RAD)
    for f, s in enumerate([1.0, 3.0, 2.0]):
        np.testing.assert_array_equal(autos[f], np.tile(np.array([s, 0, 0, 0, 0, 0, s, 0], np.float32), (3, 1)))
    # sum of flux densities (cpu.rs:506-576)
    s1 = sl.SourceComponent(*sl.radec_deg(1.0, -27.0), sl.Point(), sl.FluxList(
        [sl.FluxDensity(150e6, 1.0), sl.FluxDensity(175e6, 3.0), sl.FluxDensity(200e6, 2.0)]))
    s2 = sl.SourceComponent(*sl.radec_deg(1.1, -27.0), sl.Point(), sl.FluxList(
        [sl.FluxDensity(150e6, 0.5), sl.FluxDensity(175e6, 0.25), sl.FluxDensity(200e6, 1.5)]))
    sky2 = sl.SkyModelArrays.from_components([s1, s2])
    autos = oracle.model_autos(sky2, 3, freqs, lst, MWA_LAT_RAD)
    for f, s in enumerate([1.5, 3.25, 3.5]):
        np.testing.assert_array_equal(autos[f, :, 0], np.float32(s))
        np.testing.assert_array_equal(autos[f, :, 6], np.float32(s))


def test_shapelet_basis_table(oracle):
    tab = oracle.shapelet_basis()
    g = json.loads((GOLD / "shapelet_basis_samples.json").read_text())
    flat = tab.reshape(-1)
    # src/model/shapelets.rs:44-59
    assert not np.all(flat < np.finfo(np.float64).eps)
    assert abs(flat[10001 // 2] - 1.0) <= 1e-10
    assert abs(flat[10001 // 2 + 1] - 0.99995) <= 1e-8
    for n, i, v in g["samples_n_index_value"]:
        ours = tab[n, i]
        assert abs(ours - v) <= 1e-12 * max(1.0, abs(v)) + 1e-300, (n, i, ours, v)


def _cal_data(nt, nch, nbl, val):
    d = np.zeros((nt, nch, nbl, 8), np.float32)
    d[..., 0] = val
    d[..., 6] = val
    return d


def identity(n):
    j = np.zeros((n, 8))
    j[:, 0] = 1
    j[:, 6] = 1
    return j


def test_calibrate_trivial(oracle):
    # di_calibrate/tests.rs:37-93
    nbl = 10
    data = _cal_data(1, 1, nbl, 4.0)
    model = _cal_data(1, 1, nbl, 1.0)
    dj, r = oracle.calibrate(data, model, 0, identity(5), 20, 1e-8, 1e-5)
    assert r.converged and r.num_iterations == 10 and r.num_failed == 0 and r.max_precision < 1e-13
    np.testing.assert_allclose(dj, identity(5) * 2.0, atol=1e-14, rtol=0)


def test_calibrate_trivial_with_flags(oracle):
    # di_calibrate/tests.rs:98-235
    nbl = 10
    data = _cal_data(1, 2, nbl, 1.0)
    data[:, 0] = _cal_data(1, 1, nbl, 4.0)[:, 0]
    data[:, 1] = _cal_data(1, 1, nbl, 9.0)[:, 0]
    data[0, 0, 0, 0] = data[0, 0, 0, 6] = 9000.0
    model = _cal_data(1, 2, nbl, 1.0)
    dj0, r0 = oracle.calibrate(data, model, 0, identity(5), 20, 1e-8, 1e-5)
    dj1, r1 = oracle.calibrate(data, model, 1, identity(5), 20, 1e-8, 1e-5)
    assert r0.converged and r0.num_failed == 0 and r1.converged
    assert not np.allclose(dj0, identity(5) * 2.0)
    np.testing.assert_allclose(dj1, identity(5) * 3.0, atol=np.finfo(np.float64).eps, rtol=0)
    data[0, 0, 0] = 0
    model[0, 0, 0] = 0
    dj0, r0 = oracle.calibrate(data, model, 0, identity(5), 20, 1e-8, 1e-5)
    dj1, r1 = oracle.calibrate(data, model, 1, identity(5), 20, 1e-8, 1e-5)
    assert r0.num_iterations == 10 and r1.num_iterations == 12
    assert r0.max_precision < 1e-13 and r1.max_precision < 1e-13
    np.testing.assert_allclose(dj0, identity(5) * 2.0, atol=1e-14, rtol=0)
    np.testing.assert_allclose(dj1, identity(5) * 3.0, atol=1e-14, rtol=0)


def test_multiple_timeblocks(oracle):
    # di_calibrate/tests.rs:657-704 (three timeblocks of one timestep each)
    data = _cal_data(3, 1, 10, 4.0)
    model = _cal_data(3, 1, 10, 1.0)
    for t in range(3):
        dj, res = oracle.calibrate_timeblock(data, model, identity(5)[:, None, :], t, t + 1, 10, 1e-8, 1e-4)
        np.testing.assert_allclose(dj[:, 0], identity(5) * 2.0, atol=1e-14, rtol=0)


def test_chanblocks_without_data(oracle):
    # di_calibrate/tests.rs:706-770
    data = np.zeros((3, 1, 10, 8), np.float32)
    dj, res = oracle.calibrate_timeblock(data, data, identity(5)[:, None, :], 0, 3, 10, 1e-8, 1e-4)
    assert np.all(np.isnan(dj)) and all(r["num_iterations"] == 1 for r in res)
    one = _cal_data(3, 1, 10, 1.0)
    dj, res = oracle.calibrate_timeblock(one, one, identity(5)[:, None, :], 0, 3, 10, 1e-8, 1e-4)
    assert not np.any(np.isnan(dj)) and all(r["num_iterations"] == 1 for r in res)


def test_recalibrating_failed_chanblocks(oracle):
    # di_calibrate/tests.rs:772-844
    data = _cal_data(1, 3, 10, 4.0)
    model = _cal_data(1, 3, 10, 1.0)
    dj0 = np.repeat(identity(5)[:, None, :], 3, axis=1)
    dj0[:, 1] = 0
    dj, res = oracle.calibrate_timeblock(data, model, dj0, 0, 1, 10, 1e-8, 1e-4)
    assert [r["num_iterations"] for r in res] == [10, 2, 10]
    dj, res = oracle.calibrate_timeblock(data, model, np.zeros((5, 3, 8)), 0, 1, 10, 1e-8, 1e-4)
    assert not any(r["converged"] for r in res)


def test_list_flux_edge_cases(oracle):
    # flux_density/mod.rs:158-270: single entry (SI -0.8), exact hit, linear
    # interpolation across a sign change, extrapolation beyond the list.
    def est(fds, f):
        sky = sl.SkyModelArrays.from_components(
            [sl.SourceComponent(0.0, 0.0, sl.Point(), sl.FluxList([sl.FluxDensity(*x) for x in fds]))])
        return oracle.inst_flux(sky, [f])[0, 0, 0]

    assert est([(150e6, 2.0)], 150e6 * 2) == pytest.approx(2.0 * 2 ** -0.8, rel=1e-15)
    assert est([(100e6, 1.0), (200e6, 4.0)], 200e6) == 4.0
    assert est([(100e6, -1.0), (200e6, 1.0)], 150e6) == pytest.approx(0.0, abs=1e-15)
    si = math.log(4.0) / math.log(2.0)
    assert est([(100e6, 1.0), (200e6, 4.0)], 300e6) == pytest.approx(4.0 * 1.5 ** si, rel=1e-14)
    assert est([(100e6, 1.0), (200e6, 4.0)], 50e6) == pytest.approx(0.5 ** si, rel=1e-14)


def _c(a):
    """[...][8] -> [...][2][2] complex."""
    return (a[..., 0::2] + 1j * a[..., 1::2]).reshape(a.shape[:-1] + (2, 2))


def _mitchcal_numpy(data, model, ntiles, iters, top_then_inverse):
    """A small MitchCal on one chanblock (di_calibrate/mod.rs:640-893 without
    the stopping rules): G_p <- top_p bot_p^-1, top = sum_q D_pq G_q M_pq^H,
    bot = sum_q (M_pq G_q^H)(M_pq G_q^H)^H, averaged with the previous
    iterate every second iteration.  With top_then_inverse False the product
    is taken the other way round, bot^-1 top."""
    i, j = np.triu_indices(ntiles, 1)
    D, M = _c(data.astype(np.float64)), _c(model.astype(np.float64))  # [t][bl][2][2]
    G = np.broadcast_to(np.eye(2, dtype=complex), (ntiles, 2, 2)).copy()
    for it in range(iters):
        top = np.zeros_like(G)
        bot = np.zeros_like(G)
        for p, q, b in zip(i, j, range(len(i))):
            for t in range(D.shape[0]):
                # both directions of the baseline
                z = M[t, b] @ G[q].conj().T
                top[p] += D[t, b] @ G[q] @ M[t, b].conj().T
                bot[p] += z @ z.conj().T
                zq = M[t, b].conj().T @ G[p].conj().T
                top[q] += D[t, b].conj().T @ G[p] @ M[t, b]
                bot[q] += zq @ zq.conj().T
        new = np.stack([top[k] @ np.linalg.inv(bot[k]) if top_then_inverse else np.linalg.inv(bot[k]) @ top[k]
                        for k in range(ntiles)])
        G = 0.5 * (G + new) if it % 2 == 1 else new
    return G


def _residual(G, data, model, ntiles):
    i, j = np.triu_indices(ntiles, 1)
    D, M = _c(data.astype(np.float64)), _c(model.astype(np.float64))
    P = G[i][None] @ M @ np.conj(np.swapaxes(G[j], -1, -2))[None]
    return np.linalg.norm(P - D) / np.linalg.norm(D)


def test_mitchcal_division_order(oracle):
    """The Jones "division" of the update is top . bot^-1 (marlu's Jones /,
    di_calibrate/mod.rs:663-681).  With leaky, non-diagonal gains and a
    polarised model the two orders differ: top . bot^-1 reproduces noiseless
    data and bot^-1 . top does not; the oracle's solver reproduces the data
    as the first does."""
    rng = np.random.default_rng(21)
    ntiles, nt, nch = 8, 2, 1
    nbl = ntiles * (ntiles - 1) // 2
    model = synth.polarised_model(nt, nch, nbl, rng)
    gains = synth.truth_gains(ntiles, nch, rng, amp_sigma=0.1, leak_sigma=0.15)
    data = synth.corrupt(model, gains)
    d1, m1 = data[:, 0], model[:, 0]
    right = _residual(_mitchcal_numpy(d1, m1, ntiles, 200, True), d1, m1, ntiles)
    wrong = _residual(_mitchcal_numpy(d1, m1, ntiles, 200, False), d1, m1, ntiles)
    assert right < 1e-5 and wrong > 1e-1, (right, wrong)
    ident = np.zeros((ntiles, nch, 8))
    ident[..., 0] = ident[..., 6] = 1.0
    dj, res = oracle.calibrate_timeblock(data, model, ident, 0, nt, 200, 1e-12, 1e-4, 0)
    G = _c(dj[:, 0])
    assert _residual(G, d1, m1, ntiles) < 1e-5


def test_per_tile_beam_with_unit_gains_is_the_shared_beam():
    """The per-tile dipole-gain beam with every dipole at unit gain is the
    shared analytic beam (the array factor then separates in l and m)."""
    from oracle import oracle as O

    for az, el, f in [(0.3, 1.2, 150e6), (2.0, 0.6, 182e6), (4.1, 1.5, 200e6)]:
        ref = O.analytic_beam(az, el, f)
        sky = _one_point_sky(az, el)
        g = np.ones((1, 32))
        # a component at the given (az, el): HA/Dec from an LST of 0
        got = O.tile_beam_table(sky[0], 0, sky[1], sky[2], g, [f])[0, 0, 0]
        np.testing.assert_allclose(got, ref, rtol=0, atol=1e-12)
    # a dead dipole changes the beam, and only the row of its polarisation
    sky = _one_point_sky(1.0, 0.9)
    g = np.ones((2, 32))
    g[1, 5] = 0.0  # X dipole 5 of the second tile
    b = O.tile_beam_table(sky[0], 0, sky[1], sky[2], g, [170e6])[:, 0, 0]
    assert np.abs(b[1, 0:4] - b[0, 0:4]).max() > 1e-3
    np.testing.assert_allclose(b[1, 4:8], b[0, 4:8], rtol=0, atol=1e-15)


def _one_point_sky(az, el, lat=-0.4660608448386394):
    """A one-point sky at (az, el) for LST 0 and the given latitude."""
    import math

    from mwa_hyperdrive_b200 import srclist as sl

    # invert hd2ae: direction cosines in the (east, north, up) frame
    x = math.cos(el) * math.sin(az)
    y = math.cos(el) * math.cos(az)
    z = math.sin(el)
    # to (HA, Dec) at latitude lat
    dec = math.asin(y * math.cos(lat) + z * math.sin(lat))
    ha = math.atan2(-x, -y * math.sin(lat) + z * math.cos(lat))
    comp = sl.SourceComponent(-ha, dec, sl.Point(), sl.PowerLaw(-0.8, sl.FluxDensity(150e6, 1.0)))
    return sl.SkyModelArrays.from_components([comp]), 0.0, lat
