"""Visibility preparation on the device (hdc_vis_average,
hdc_scale_by_weights) against the oracle's restatements of vis_average
(averaging/mod.rs:537-648) and CalVis::scale_by_weights
(params/di_calibration.rs:578-625): bit for bit, since both are FP64 sums
and products in the reference's order rounded once to FP32."""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("no CUDA device", allow_module_level=True)

from mwa_hyperdrive_b200 import _lib  # noqa: E402
from mwa_hyperdrive_b200 import calibrate as cal  # noqa: E402


def mixed_weights(rng, shape):
    """Positive, zero and negative (flagged) weights, with whole
    (timestep, channel) rows flagged for some baselines."""
    w = rng.uniform(0.1, 20.0, size=shape).astype(np.float32)
    u = rng.uniform(size=shape)
    w[u < 0.1] = 0.0
    w[(u >= 0.1) & (u < 0.25)] *= -1.0
    w[:, :, ::7] = -np.abs(w[:, :, ::7])  # every 7th baseline fully flagged
    return w


@pytest.mark.parametrize("nt,nf,nbl,nout,flagged", [
    (1, 4, 1, 4, ()),
    (2, 3, 1, 2, ()),
    (4, 64, 8128, 4, ()),
    (2, 48, 8128, 22, (0, 23)),
    (3, 7, 33, 3, (1,)),
    (8, 32, 2016, 1, ()),
    (2, 1200, 64, 300, tuple(range(598, -1, -2))),  # more than 256 flagged, given in descending order
])
def test_vis_average_matches_oracle(oracle, nt, nf, nbl, nout, flagged):
    rng = np.random.default_rng(nt * 1000 + nf)
    v = rng.normal(size=(nt, nf, nbl, 8)).astype(np.float32)
    w = mixed_weights(rng, (nt, nf, nbl))
    exp, wexp = oracle.vis_average(v, w, nout, flagged)
    to, wto = cal.vis_average(torch.from_numpy(v).cuda(), torch.from_numpy(w).cuda(), nout, flagged)
    np.testing.assert_array_equal(to.cpu().numpy(), exp)
    np.testing.assert_array_equal(wto.cpu().numpy(), wexp)


def test_vis_average_known_answers():
    """averaging/tests.rs:562-679: 2 timesteps x 4 channels of identity x 1..8
    with prime weights; averaged per channel and in pairs of channels."""
    ident = np.array([1, 0, 0, 0, 0, 0, 1, 0], np.float32)
    v = (np.arange(1, 9, dtype=np.float32).reshape(2, 4, 1, 1) * ident).astype(np.float32)
    w = np.array([[[2.0], [3.0], [5.0], [7.0]], [[11.0], [13.0], [17.0], [19.0]]], np.float32)
    dv, dw = torch.from_numpy(v).cuda(), torch.from_numpy(w).cuda()
    to, wto = cal.vis_average(dv, dw, 4)
    np.testing.assert_allclose(to.cpu().numpy()[:, 0, 0], [57 / 13, 84 / 16, 134 / 22, 180 / 26], rtol=1e-7)
    np.testing.assert_array_equal(wto.cpu().numpy()[:, 0], [13, 16, 22, 26])
    to, wto = cal.vis_average(dv, dw, 2)
    np.testing.assert_allclose(to.cpu().numpy()[:, 0, 0], [(57 + 84) / 29, (134 + 180) / 48], rtol=1e-7)
    np.testing.assert_array_equal(wto.cpu().numpy()[:, 0], [29, 48])
    w[:, 0] *= -1
    to, wto = cal.vis_average(dv, torch.from_numpy(w).cuda(), 4)
    assert to.cpu().numpy()[0, 0, 0] == 3.0 and wto.cpu().numpy()[0, 0] == -13.0


def test_vis_average_rejects_bad_chunks():
    v = torch.zeros((1, 6, 2, 8), device="cuda")
    w = torch.ones((1, 6, 2), device="cuda")
    with pytest.raises(_lib.HdcError):
        cal.vis_average(v, w, 2, (1, 1))
    with pytest.raises(_lib.HdcError):
        cal.vis_average(v, w, 2, (5,))
    with pytest.raises(_lib.HdcError):
        cal.vis_average(v, w, 5)  # 6 channels make chunks of 2: only 3 of them


@pytest.mark.parametrize("with_baseline_weights", [False, True])
def test_scale_by_weights_matches_oracle(oracle, with_baseline_weights):
    rng = np.random.default_rng(3)
    nt, nch, nbl = 3, 24, 8128
    d = rng.normal(size=(nt, nch, nbl, 8)).astype(np.float32)
    m = rng.normal(size=(nt, nch, nbl, 8)).astype(np.float32)
    w = mixed_weights(rng, (nt, nch, nbl))
    bw = None
    if with_baseline_weights:
        bw = rng.uniform(0.0, 1.5, size=nbl)
        bw[::11] = 0.0
    exp_d, exp_m = oracle.scale_by_weights(d, m, w, bw)
    dd, dm = torch.from_numpy(d).cuda(), torch.from_numpy(m).cuda()
    cal.scale_by_weights(dd, dm, torch.from_numpy(w).cuda(), bw)
    np.testing.assert_array_equal(dd.cpu().numpy(), exp_d)
    np.testing.assert_array_equal(dm.cpu().numpy(), exp_m)
