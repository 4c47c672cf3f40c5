"""model_points_noalloc, the point-source predict for callers that cannot
allocate device memory (hosts that keep the whole GPU under their own memory
pool, or loops that must not call cudaMalloc and its implicit device
synchronisation).  It must give the same visibilities as model_points, twice
in a row on the shared fixed scratch, without changing the device's free
memory; match the FP64 oracle; report a kernel's timed-out wait and start the
next call clean; and refuse problems larger than its fixed scratch.

This file is collected last on purpose, so that a run that stops at the first
failure has already run every other test.
"""

import ctypes
import math

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("no CUDA device", allow_module_level=True)

from mwa_hyperdrive_b200 import _lib  # noqa: E402
from mwa_hyperdrive_b200 import srclist as sl  # noqa: E402
from mwa_hyperdrive_b200 import synth  # noqa: E402


def assert_f32_close(a, b, ulps=4):
    # the tolerance the other drop-in predictor tests use
    a = np.asarray(a, np.float32)
    b = np.asarray(b, np.float32)
    scale = np.maximum(np.abs(b), np.float32(np.max(np.abs(b)) * 1e-6 + 1e-30))
    bad = np.abs(a - b) > ulps * np.spacing(scale)
    assert not bad.any(), f"{bad.sum()} elements differ; max diff {np.max(np.abs(a - b))}"


class PointsProblem:
    """Device tables of the reference's Points / Addresses for a random
    point-source sky: 3 power laws, 3 curved power laws, 3 list fluxes, with
    per-tile beam Jones (3 unique tiles, 2 unique channels)."""

    def __init__(self, seed, ntiles=21, nf=6):
        rng = np.random.default_rng(seed)
        self.pc = (0.2, math.radians(-28.0))
        self.xyzs = synth.tiles_in_disk(ntiles, 1200.0, seed)
        self.freqs = 150e6 + np.arange(nf) * 1.28e6
        self.nbl = ntiles * (ntiles - 1) // 2
        self.nf = nf
        pos = synth.cap_positions(9, self.pc, math.radians(6.0), rng)
        # instrumental flux at 150 MHz and lists, built directly (XX, XY, YX, YY)
        fds = np.zeros((9, 8))
        fds[:, 0] = rng.uniform(0.5, 3.0, 9)
        fds[:, 6] = fds[:, 0] * 0.9
        fds[:, 2] = 0.05
        fds[:, 4] = 0.05
        lists = np.zeros((nf, 3, 8))
        lists[..., 0] = rng.uniform(0.5, 2.0, (nf, 3))
        lists[..., 6] = lists[..., 0]
        lmn = np.zeros((9, 3))
        for k in range(9):
            ra, dec = pos[k]
            d_ra = ra - self.pc[0]
            l = math.cos(dec) * math.sin(d_ra)
            m = math.sin(dec) * math.cos(self.pc[1]) - math.cos(dec) * math.sin(self.pc[1]) * math.cos(d_ra)
            n = math.sin(dec) * math.sin(self.pc[1]) + math.cos(dec) * math.cos(self.pc[1]) * math.cos(d_ra)
            lmn[k] = [2 * math.pi * l, 2 * math.pi * m, 2 * math.pi * (n - 1)]
        beam = rng.normal(size=(3, 2, 9, 8)) * 0.2
        beam[..., 0] += 1.0
        beam[..., 6] += 1.0
        ha = 0.21 - self.pc[0]
        s_ha, c_ha, s_d, c_d = math.sin(ha), math.cos(ha), math.sin(self.pc[1]), math.cos(self.pc[1])
        tuvw = np.stack([s_ha * self.xyzs[:, 0] + c_ha * self.xyzs[:, 1],
                         -s_d * c_ha * self.xyzs[:, 0] + s_d * s_ha * self.xyzs[:, 1] + c_d * self.xyzs[:, 2],
                         c_d * c_ha * self.xyzs[:, 0] - c_d * s_ha * self.xyzs[:, 1] + s_d * self.xyzs[:, 2]], -1)
        i, j = np.triu_indices(ntiles, 1)
        uvws = tuvw[i] - tuvw[j]
        self.keep = {}

        def put(name, arr, dt=np.float64):
            t = torch.from_numpy(np.ascontiguousarray(arr, dt)).cuda()
            self.keep[name] = t
            return t.data_ptr()

        lm = put("lmn", lmn)
        fd = put("fds", fds)
        sis = put("sis", rng.normal(-0.8, 0.2, 6))
        qs = put("qs", rng.normal(0.0, 0.1, 3))
        lf = put("lists", lists)
        self.points = _lib.Points(3, lm, fd, sis, 3, lm + 72, fd + 192, sis + 24, qs, 3, lm + 144, lf)
        self.addr = _lib.Addresses(nf, nf * self.nbl, self.nbl, put("freqs", self.freqs), 0, 2,
                                   put("tm", np.arange(ntiles) % 3, np.int32),
                                   put("fm", np.arange(nf) * 2 // nf, np.int32),
                                   put("um", np.arange(ntiles), np.int32))
        self.uvws = put("uvws", uvws)
        self.beam = put("beam", beam)

    def run(self, fn_name):
        vis = torch.zeros((self.nf, self.nbl, 8), dtype=torch.float32, device="cuda")
        fn = getattr(_lib.lib(), fn_name)
        res = fn(ctypes.byref(self.points), ctypes.byref(self.addr), self.uvws, self.beam, vis.data_ptr())
        _lib.check_str(res, fn_name)
        torch.cuda.synchronize()
        return vis.cpu().numpy()


def test_noalloc_matches_model_points_twice():
    first = PointsProblem(seed=1)
    second = PointsProblem(seed=2, ntiles=17, nf=9)
    ref1 = first.run("model_points")
    ref2 = second.run("model_points")
    got1 = first.run("model_points_noalloc")
    assert_f32_close(got1, ref1)
    # the second call reuses the shared scratch with a different problem size
    free_before = torch.cuda.mem_get_info()[0]
    got2 = second.run("model_points_noalloc")
    free_after = torch.cuda.mem_get_info()[0]
    assert_f32_close(got2, ref2)
    assert free_after == free_before
    # and the first problem again, after the second overwrote the scratch
    assert_f32_close(first.run("model_points_noalloc"), ref1)


class OracleProblem:
    """A point-source sky (power laws, curved power laws, lists) as the
    reference's Points / Addresses device tables with a per-tile beam (3
    unique tiles, 2 unique channels), and the oracle's visibilities for it."""

    def __init__(self, oracle, seed=7, ntiles=14, nf=5):
        rng = np.random.default_rng(seed)
        obs = synth.Obs(synth.tiles_in_disk(ntiles, 1000.0, seed), 150e6 + np.arange(nf) * 1.28e6,
                        (0.2, math.radians(-28.0)), np.array([0.25]))
        pc, lst = obs.phase_centre, obs.lsts[0]
        pos = synth.cap_positions(9, pc, math.radians(6.0), rng)
        comps = []
        for k in range(9):
            fd = sl.FluxDensity(150e6, float(rng.uniform(0.5, 3.0)), 0.1, -0.05, 0.02)
            ft = [sl.PowerLaw(-0.7, fd), sl.CurvedPowerLaw(-0.9, fd, 0.1),
                  sl.FluxList([sl.FluxDensity(140e6, 2.0), sl.FluxDensity(190e6, 1.0)])][k // 3]
            comps.append(sl.SourceComponent(float(pos[k, 0]), float(pos[k, 1]), sl.Point(), ft))
        sky = sl.SkyModelArrays.from_components(comps)
        nt, self.nf, self.nbl = ntiles, nf, obs.num_baselines
        uvws = oracle.xyzs_to_cross_uvws(obs.tile_xyzs, lst - pc[0], pc[1])
        tile_map = (np.arange(nt) % 3).astype(np.int32)
        freq_map = (np.arange(nf) * 2 // nf).astype(np.int32)
        beam = rng.normal(size=(3, 2, 9, 8)) * 0.3
        beam[..., 0] += 1.0
        beam[..., 6] += 1.0
        lmn = np.array([oracle.lmn_rime(c.ra, c.dec, *pc) for c in comps])
        inst150 = oracle.inst_flux(sky, [150e6])[0]
        list_fds = oracle.inst_flux(sky, obs.freqs)[:, 6:9]
        self.keep = []

        def put(arr, dt=np.float64):
            t = torch.from_numpy(np.ascontiguousarray(arr, dt)).cuda()
            self.keep.append(t)
            return t.data_ptr()

        lm, fd_p, sis = put(lmn), put(inst150), put([-0.7] * 3 + [-0.9] * 3)
        self.points = _lib.Points(3, lm, fd_p, sis, 3, lm + 72, fd_p + 192, sis + 24, put([0.1] * 3), 3, lm + 144,
                                  put(list_fds))
        self.addr = _lib.Addresses(nf, nf * self.nbl, self.nbl, put(obs.freqs), 0, 2, put(tile_map, np.int32),
                                   put(freq_map, np.int32), put(np.arange(nt), np.int32))
        self.uvws, self.beam = put(uvws), put(beam)
        b = oracle.beam_struct(2, [beam, None, None], tile_map, freq_map, 2)
        self.ref = oracle.model_type(0, sky, obs.tile_xyzs, obs.freqs, pc, lst, synth.MWA_LAT_RAD, uvws, beam=b)

    def call(self, fn_name, vis):
        fn = getattr(_lib.lib(), fn_name)
        return fn(ctypes.byref(self.points), ctypes.byref(self.addr), self.uvws, self.beam, vis.data_ptr())


def test_noalloc_against_the_oracle_and_after_a_timeout(oracle):
    """The same call checked against the FP64 oracle (f32 output within the
    drop-in tests' 4 ulps); a kernel whose bounded wait runs out (the test
    hook makes the next predict kernel issue no table copies and wait 1 ms)
    must give an error string and leave the visibilities unchanged, and the
    call after it must start from a clear error word and be right again."""
    prob = OracleProblem(oracle)
    vis = torch.zeros((prob.nf, prob.nbl, 8), dtype=torch.float32, device="cuda")
    _lib.check_str(prob.call("model_points_noalloc", vis), "model_points_noalloc")
    torch.cuda.synchronize()
    assert_f32_close(vis.cpu().numpy(), prob.ref)
    vis.fill_(0.5)
    assert _lib.lib().hdc_test_stall_next_predict(1_000_000) == 0
    res = prob.call("model_points_noalloc", vis)
    assert res is not None and b"bounded wait ran out" in res
    torch.cuda.synchronize()
    assert torch.all(vis == 0.5)
    vis.zero_()
    _lib.check_str(prob.call("model_points_noalloc", vis), "model_points_noalloc")
    torch.cuda.synchronize()
    assert_f32_close(vis.cpu().numpy(), prob.ref)


def test_noalloc_rejects_problems_beyond_its_scratch():
    # 4000 channels x 90 components need ~23 MB > 16 MiB; the call must fail
    # on the host before launching anything (no device pointer is touched).
    pts = _lib.Points(90, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0)
    addr = _lib.Addresses(4000, 4000 * 10, 10, 0, 0, 1, 0, 0, 0)
    vis = torch.zeros(8, dtype=torch.float32, device="cuda")
    res = _lib.lib().model_points_noalloc(ctypes.byref(pts), ctypes.byref(addr), 0, 0, vis.data_ptr())
    assert res is not None and b"16 MiB" in res
