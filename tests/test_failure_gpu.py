"""Failure paths on the GPU, exercised in forms that fault nothing.

* A bounded wait that runs out: hdc_test_stall_next_predict makes the next
  direct predict kernel issue none of its table copies and wait only a
  millisecond, so the wait runs out with nothing in flight.  The drop-in call
  must return the timeout string and leave the visibilities unchanged, the
  native modeller must return HDC_ERR_TIMEOUT (the host-buffer call at once,
  the asynchronous device call at the next call), and the next call must
  succeed with the right answer.
* A failed device allocation: a drop-in call whose derived tables need far
  more memory than the GPU has (the reference's gpu/tests.rs:26-40 asks
  cudaMalloc for 1 TB) must return an error string, and the library must work
  afterwards.
* NaN inputs to DI calibration: a tile whose baselines are all NaN, a single
  NaN visibility and an all-NaN model chanblock must give the oracle's
  iteration counts, failed-tile counts and NaN patterns
  (di_calibrate/mod.rs:754-784 failed tiles, :770-773 NaN solutions).
"""

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
from mwa_hyperdrive_b200 import calibrate as cal  # noqa: E402
from mwa_hyperdrive_b200.model import SkyModeller  # noqa: E402

STALL_NS = 1_000_000  # 1 ms: the stalled wait's limit


class DropinPoints:
    """The reference's Points / Addresses device tables for a small random
    point-source sky of power laws (no beam)."""

    def __init__(self, oracle, ntiles=16, nf=5, nc=70, seed=3):
        rng = np.random.default_rng(seed)
        obs = synth.Obs(synth.tiles_in_disk(ntiles, 900.0, seed), 160e6 + np.arange(nf) * 1.28e6,
                        (0.3, math.radians(-27.0)), np.array([0.35]))
        pos = synth.cap_positions(nc, obs.phase_centre, math.radians(8.0), rng)
        comps = [sl.SourceComponent(float(pos[k, 0]), float(pos[k, 1]), sl.Point(),
                                    sl.PowerLaw(float(rng.normal(-0.8, 0.2)),
                                                sl.FluxDensity(150e6, float(rng.lognormal(0.0, 1.0)))))
                 for k in range(nc)]
        sky = sl.SkyModelArrays.from_components(comps)
        pc, lst = obs.phase_centre, obs.lsts[0]
        self.nf, self.nbl, self.nc = nf, obs.num_baselines, nc
        uvws = oracle.xyzs_to_cross_uvws(obs.tile_xyzs, lst - pc[0], pc[1])
        lmn = np.array([oracle.lmn_rime(c.ra, c.dec, *pc) for c in comps])
        inst150 = oracle.inst_flux(sky, [150e6])[0]
        self.keep = []

        def put(arr, dt=np.float64):
            t = torch.from_numpy(np.ascontiguousarray(arr, dt)).cuda()
            self.keep.append(t)
            return t.data_ptr()

        self.points = _lib.Points(nc, put(lmn), put(inst150), put([c.flux_type.si for c in comps]), 0, 0, 0, 0, 0, 0, 0,
                                  0)
        self.addr = _lib.Addresses(nf, nf * self.nbl, self.nbl, put(obs.freqs), 0, 0, 0, 0, 0)
        self.uvws = put(uvws)
        self.ref = oracle.model_type(0, sky, obs.tile_xyzs, obs.freqs, pc, lst, synth.MWA_LAT_RAD, uvws)

    def call(self, vis):
        return _lib.lib().model_points(ctypes.byref(self.points), ctypes.byref(self.addr), self.uvws, None,
                                       vis.data_ptr())


def assert_f32_close(a, b, ulps=4):
    a, b = np.asarray(a, np.float32), np.asarray(b, np.float32)
    scale = np.maximum(np.abs(b), np.float32(np.max(np.abs(b)) * 1e-6 + 1e-30))
    bad = np.abs(a - b) > ulps * np.spacing(scale)
    assert not bad.any(), f"{bad.sum()} elements differ; max diff {np.max(np.abs(a - b))}"


def test_dropin_timeout_is_reported_and_cleared(oracle):
    prob = DropinPoints(oracle)
    start = torch.full((prob.nf, prob.nbl, 8), 0.25, dtype=torch.float32, device="cuda")
    vis = start.clone()
    assert _lib.lib().hdc_test_stall_next_predict(STALL_NS) == 0
    res = prob.call(vis)
    assert res is not None and b"bounded wait ran out" in res
    assert b"model_points" in _lib.lib().hdc_last_error()
    torch.cuda.synchronize()
    # no CTA added a partial sum
    assert torch.equal(vis, start)
    # the word was cleared: the next call succeeds and is right
    vis.zero_()
    _lib.check_str(prob.call(vis), "model_points")
    torch.cuda.synchronize()
    assert_f32_close(vis.cpu().numpy(), prob.ref, ulps=4)


def small_modeller(form="direct"):
    obs, sky = synth.config1()
    freqs = obs.freqs[:6]
    return SkyModeller(sky, obs.tile_xyzs, freqs, obs.phase_centre, obs.latitude, form=form), obs, freqs


def test_modeller_host_call_reports_its_own_timeout():
    m, obs, freqs = small_modeller()
    ref = np.zeros((freqs.size, obs.num_baselines, 8), np.float32)
    m.model_timestep_with_host(obs.lsts[0], ref)
    _lib.lib().hdc_test_stall_next_predict(STALL_NS)
    vis = np.zeros_like(ref)
    with pytest.raises(_lib.HdcError, match=r"status 4\).*bounded wait ran out"):
        m.model_timestep_with_host(obs.lsts[0], vis)
    # the stalled launch (the first channel chunk) left its channels unchanged
    assert np.all(vis[0] == 0.0)
    vis = np.zeros_like(ref)
    m.model_timestep_with_host(obs.lsts[0], vis)
    np.testing.assert_array_equal(vis, ref)


def test_modeller_device_call_timeout_surfaces_at_next_call():
    m, obs, freqs = small_modeller()
    vis = torch.zeros((freqs.size, obs.num_baselines, 8), dtype=torch.float32, device="cuda")
    m.model_timestep_with(obs.lsts[0], vis, return_uvws=False)
    torch.cuda.synchronize()
    ref = vis.clone()
    _lib.lib().hdc_test_stall_next_predict(STALL_NS)
    vis.zero_()
    # asynchronous: the call itself cannot know yet
    m.model_timestep_with(obs.lsts[0], vis, return_uvws=False)
    torch.cuda.synchronize()
    assert torch.all(vis == 0)
    with pytest.raises(_lib.HdcError, match=r"status 4\)"):
        m.model_timestep_with(obs.lsts[0], vis, return_uvws=False)
    # reported once: the following call is clean and right
    vis.zero_()
    m.model_timestep_with(obs.lsts[0], vis, return_uvws=True)
    torch.cuda.synchronize()
    assert torch.equal(vis, ref)


def test_failed_device_allocation_is_an_error_not_a_crash(oracle):
    # 200 000 channels x 100 000 components of derived flux tables = 1.3 TB:
    # the scratch allocation fails before any kernel reads the (null) tables
    pts = _lib.Points(100_000, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0)
    addr = _lib.Addresses(200_000, 200_000 * 10, 10, 0, 0, 0, 0, 0, 0)
    vis = torch.zeros(8, dtype=torch.float32, device="cuda")
    res = _lib.lib().model_points(ctypes.byref(pts), ctypes.byref(addr), 0, 0, vis.data_ptr())
    assert res is not None and b"out of device memory" in res
    assert b"allocation" in _lib.lib().hdc_last_error()
    # the library still works
    prob = DropinPoints(oracle, seed=4)
    vis = torch.zeros((prob.nf, prob.nbl, 8), dtype=torch.float32, device="cuda")
    _lib.check_str(prob.call(vis), "model_points")
    torch.cuda.synchronize()
    assert_f32_close(vis.cpu().numpy(), prob.ref, ulps=4)


def identity(n, nch):
    j = np.zeros((n, nch, 8))
    j[..., 0] = j[..., 6] = 1.0
    return j


@pytest.mark.parametrize("form", ["plain", "collapsed"])
def test_nan_inputs_follow_the_reference(oracle, form):
    rng = np.random.default_rng(5)
    ntiles, nt, nch = 12, 2, 4
    nbl = ntiles * (ntiles - 1) // 2
    model = synth.random_model(nt, nch, nbl, rng)
    data = synth.corrupt(model, synth.truth_gains(ntiles, nch, rng), rng, 20.0)
    i, j = np.triu_indices(ntiles, 1)
    data[:, 1, (i == 3) | (j == 3)] = np.nan  # every baseline of tile 3 in chanblock 1
    data[0, 2, 5, 0] = np.nan  # one visibility of chanblock 2
    model[:, 3] = np.nan  # the whole model of chanblock 3
    dj_o, res_o = oracle.calibrate_timeblock(data, model, identity(ntiles, nch), 0, nt, 50, 1e-8, 1e-4, 0)
    dj = torch.from_numpy(identity(ntiles, nch)).cuda()
    res = cal.calibrate_timeblock(torch.from_numpy(data).cuda(), torch.from_numpy(model).cuda(), dj, (0, nt), 50,
                                  1e-8, 1e-4, form=form)
    dj_g = dj.cpu().numpy()
    assert [r.num_iterations for r in res] == [r["num_iterations"] for r in res_o]
    assert [r.converged for r in res] == [r["converged"] for r in res_o]
    assert [r.num_failed for r in res] == [r["num_failed"] for r in res_o]
    np.testing.assert_array_equal(np.isnan(dj_g), np.isnan(dj_o))
    ok = ~np.isnan(dj_o)
    tol = 1e-10 if form == "plain" else 1e-9
    assert np.linalg.norm(dj_g[ok] - dj_o[ok]) / np.linalg.norm(dj_o[ok]) < tol
