"""From a uvfits file to DI solutions on the GPU: visibilities written by
write_uvfits and read back by UvfitsReader (both baseline conventions) go
through vis_average and the DI solver, and must give what the same arrays
give without the file, and the CPU oracle's solutions."""

import math

import numpy as np
import pytest

from mwa_hyperdrive_b200 import synth
from mwa_hyperdrive_b200 import uvfits as U
from oracle import oracle as O

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("no CUDA device", allow_module_level=True)

from mwa_hyperdrive_b200 import calibrate as cal  # noqa: E402


@pytest.mark.parametrize("ant2_minus_ant1", [False, True])
def test_uvfits_to_solutions(tmp_path, ant2_minus_ant1):
    rng = np.random.default_rng(11)
    ntiles, nt, nch = 16, 2, 6
    nbl = ntiles * (ntiles - 1) // 2
    model = synth.random_model(nt, nch, nbl, rng)
    data = synth.corrupt(model, synth.truth_gains(ntiles, nch, rng), rng, 40.0).astype(np.float32)
    wts = np.ones((nt, nch, nbl), np.float32)
    xyz = synth.tiles_in_disk(ntiles, 800.0, 4)
    jds = np.array([U.gps_to_jd_utc(1090008658.0 + 8.0 * t) for t in range(nt)])
    freqs = 167.0e6 + 40e3 * np.arange(nch)
    pos = (math.radians(116.67), math.radians(-26.70), 377.0)
    p = tmp_path / "obs.uvfits"
    U.write_uvfits(p, data, wts, jds, freqs, [f"T{i}" for i in range(ntiles)], xyz, pos, (0.0, math.radians(-27.0)),
                   ant2_minus_ant1=ant2_minus_ant1)
    r = U.UvfitsReader(p)
    read = np.stack([r.read_crosses(t)[0] for t in range(nt)])
    rw = np.stack([r.read_crosses(t)[1] for t in range(nt)])
    np.testing.assert_array_equal(read, data)

    # the timeblock averaged to one chanblock per channel on the device, as
    # the reference does before calibrating, against the oracle
    d_read = torch.from_numpy(read).cuda()
    d_w = torch.from_numpy(rw).cuda()
    avg, wavg = cal.vis_average(d_read, d_w, nch)
    exp, wexp = O.vis_average(read, rw, nch)
    np.testing.assert_array_equal(avg.cpu().numpy(), exp)
    np.testing.assert_array_equal(wavg.cpu().numpy(), wexp)

    start = np.zeros((ntiles, nch, 8))
    start[..., 0] = start[..., 6] = 1.0
    sols = []
    for vis in (read, data):
        dj = torch.from_numpy(start.copy()).cuda()
        cal.calibrate_timeblock(torch.from_numpy(np.ascontiguousarray(vis)).cuda(),
                                torch.from_numpy(model.astype(np.float32)).cuda(), dj, (0, nt), 200, 1e-8, 1e-4,
                                form="plain")
        sols.append(dj.cpu().numpy())
    # the same inputs: equal up to the order of the solver's shared-memory
    # atomic sums (not fixed from run to run)
    np.testing.assert_allclose(sols[0], sols[1], rtol=1e-12, atol=1e-15)
    ref, _ = O.calibrate_timeblock(data.astype(np.float64), model.astype(np.float32).astype(np.float64), start, 0, nt,
                                   200, 1e-8, 1e-4, 0)
    fin = np.isfinite(ref)
    assert np.array_equal(np.isfinite(sols[0]), fin)
    assert np.max(np.abs(sols[0][fin] - ref[fin])) <= 1e-9 * np.max(np.abs(ref[fin]))
