"""into_cal_sols on the device (hdc_into_cal_sols) against the oracle's
restatement of di_calibrate/mod.rs:89-262: inversion (marlu Jones::inv, or
Complex::inv of XX / YY alone), NaN padding of flagged tiles and
chanblocks, and the host padding of precisions and baseline weights; then a
write/read round trip of the completed solutions."""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("no CUDA device", allow_module_level=True)

from mwa_hyperdrive_b200 import _lib  # noqa: E402
from mwa_hyperdrive_b200 import solutions as S  # noqa: E402
from mwa_hyperdrive_b200.model import POLS  # noqa: E402


def gains(rng, shape):
    g = rng.normal(size=shape + (8,))
    g[..., 0] += 3.0  # well away from singular
    g[..., 6] += 3.0
    return g


def same(a, b):
    """Bit-identical, NaNs included."""
    assert a.shape == b.shape
    assert np.array_equal(np.isnan(a), np.isnan(b))
    m = ~np.isnan(a)
    np.testing.assert_array_equal(a[m], b[m])


@pytest.mark.parametrize("pols", list(POLS))
@pytest.mark.parametrize("ntb,nut,nuc,ft,fc", [
    (1, 126, 764, [3, 77], [0, 383, 384, 767]),
    (3, 8, 5, [], []),
    (2, 1, 1, [0, 2], [1]),
    (1, 120, 300, list(range(0, 128, 16)), list(range(0, 600, 2))),
])
def test_into_cal_sols_matches_oracle(oracle, pols, ntb, nut, nuc, ft, fc):
    rng = np.random.default_rng(ntb * 7 + nut)
    dj = gains(rng, (ntb, nut, nuc))
    exp = oracle.into_cal_sols(dj, ft, fc, POLS[pols])
    got = S.into_cal_sols_device(torch.from_numpy(dj).cuda(), ft[::-1], fc[::-1], pols).cpu().numpy()
    same(got, exp)


def test_into_cal_sols_pads_results_and_weights():
    rng = np.random.default_rng(2)
    ntiles, ft, fc = 6, [1, 4], [2]
    nut, nuc = ntiles - len(ft), 5
    dj = gains(rng, (2, nut, nuc))
    res = rng.uniform(size=(2, nuc))
    nbl_u = nut * (nut - 1) // 2
    bw = np.arange(1.0, nbl_u + 1)
    s = S.into_cal_sols(torch.from_numpy(dj).cuda(), ft, fc, calibration_results=res, unflagged_baseline_weights=bw,
                        max_iterations=50, stop_threshold=1e-8, min_threshold=1e-4)
    assert s.di_jones.shape == (2, ntiles, nuc + 1, 8)
    assert np.isnan(s.di_jones[:, [1, 4]]).all() and np.isnan(s.di_jones[:, :, 2]).all()
    assert np.isnan(s.calibration_results[:, 2]).all()
    np.testing.assert_array_equal(s.calibration_results[:, [0, 1, 3, 4, 5]], res)
    k, exp = 0, []
    for t1 in range(ntiles):
        for t2 in range(t1 + 1, ntiles):
            if t1 in ft or t2 in ft:
                exp.append(np.nan)
            else:
                k += 1
                exp.append(float(k))
    np.testing.assert_array_equal(np.isnan(s.baseline_weights), np.isnan(exp))
    np.testing.assert_array_equal(s.baseline_weights[~np.isnan(exp)], np.array(exp)[~np.isnan(exp)])
    assert s.flagged_tiles == ft and s.flagged_chanblocks == fc


def test_completed_solutions_round_trip(tmp_path):
    rng = np.random.default_rng(4)
    dj = gains(rng, (1, 10, 12))
    s = S.into_cal_sols(torch.from_numpy(dj).cuda(), [3], [0, 7], calibration_results=np.full((1, 12), 1e-9),
                        tile_names=[f"Tile{i:03d}" for i in range(11)])
    for ext in ("fits", "bin"):
        p = tmp_path / f"s.{ext}"
        S.write_solutions(s, p)
        r = S.read_solutions(p)
        same(r.di_jones, s.di_jones)
        assert r.flagged_tiles == [3] and r.flagged_chanblocks == [0, 7]


def test_rejects_bad_flags():
    d = torch.zeros((1, 2, 2, 8), dtype=torch.float64, device="cuda")
    with pytest.raises(_lib.HdcError):
        S.into_cal_sols_device(d, [1, 1], [])
    with pytest.raises(_lib.HdcError):
        S.into_cal_sols_device(d, [], [9])
