"""Learned warm start: the MLP's CUDA gradients against the float64 numpy
oracle, training on solver-produced solutions, the judge-and-fallback rule,
and what the trained network gains over the identity start."""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("no CUDA device", allow_module_level=True)

from mwa_hyperdrive_b200 import calibrate as cal  # noqa: E402
from mwa_hyperdrive_b200 import warmstart as ws  # noqa: E402
from oracle import mlp_ref  # noqa: E402


def test_gradients_match_numpy_oracle():
    rng = np.random.default_rng(0)
    m = ws.WarmStartMLP(hidden=48, num_hidden=3, seed=3)
    p = m.get_params()
    # give the (zero-initialised) output layer values so every gradient is exercised
    p = p + rng.normal(0, 0.05, p.size).astype(np.float32)
    m.set_params(p)
    x = rng.normal(size=(300, ws.IN_DIM)).astype(np.float32)
    t = rng.normal(size=(300, ws.OUT_DIM)).astype(np.float32)
    loss, g = m.gradients(torch.from_numpy(x).cuda(), torch.from_numpy(t).cuda())
    ref_loss, ref_g = mlp_ref.gradients(p, m.dims, x, t, ws.CENTRE)
    assert abs(loss - ref_loss) <= 1e-5 * ref_loss
    err = np.linalg.norm(g - ref_g) / np.linalg.norm(ref_g)
    assert err < 1e-5, err
    y = torch.empty((300, ws.OUT_DIM), device="cuda")
    m.forward_device(torch.from_numpy(x).cuda(), y)
    yr, _ = mlp_ref.forward(p, m.dims, x, ws.CENTRE)
    np.testing.assert_allclose(y.cpu().numpy(), yr, rtol=1e-4, atol=1e-5)


def test_training_reduces_loss():
    rng = np.random.default_rng(1)
    m = ws.WarmStartMLP(hidden=64, num_hidden=2, seed=1)
    x = rng.normal(size=(8192, ws.IN_DIM)).astype(np.float32)
    # target: centre input plus a smooth function of the neighbours
    y = x[:, ws.CENTRE:ws.CENTRE + 8] + 0.3 * np.tanh(x[:, :8] - x[:, 32:40])
    losses = m.train(x, y.astype(np.float32), epochs=30, batch=1024, lr=2e-3)
    assert losses[-1] < 0.2 * losses[0], losses


def test_save_load_roundtrip(tmp_path):
    m = ws.WarmStartMLP(hidden=32, num_hidden=3, seed=5)
    p = m.get_params() + 0.01
    m.set_params(p)
    m.save(tmp_path / "w.bin")
    m2 = ws.WarmStartMLP.load(tmp_path / "w.bin")
    np.testing.assert_array_equal(m2.get_params(), p.astype(np.float32))
    raw = bytearray((tmp_path / "w.bin").read_bytes())
    raw[20] ^= 1
    (tmp_path / "bad.bin").write_bytes(bytes(raw))
    with pytest.raises(ValueError):
        ws.WarmStartMLP.load(tmp_path / "bad.bin")


def solve_sequence(blocks, mlp, tight):
    """Solve consecutive timeblocks; timeblock k>0 starts from the judged MLP
    proposal (mlp) or identity (mlp None).  Returns solutions, iterations."""
    prev = None
    sols, iters, chose = [], [], []
    for data, model, _ in blocks:
        d = torch.from_numpy(data).cuda()
        m = torch.from_numpy(model).cuda()
        sol, res, use, _ = ws.calibrate_warm(d, m, (0, data.shape[0]), prev, mlp, max_iterations=tight[0],
                                             stop_threshold=tight[1], min_threshold=1e-4)
        sols.append(sol.cpu().numpy())
        iters.append(np.array([r.num_iterations for r in res]))
        chose.append(use.cpu().numpy().astype(bool) if use is not None else np.zeros(data.shape[1], bool))
        prev = sol
    return sols, iters, chose


def test_trained_warm_start_halves_iterations_to_the_same_solutions():
    """Both arms run the unchanged MitchCal iteration to stop 1e-15 (tight
    enough that each lands within 1e-6 of the solver's fixed point: the
    iteration converges linearly, and at the default stop 1e-8 a solution can
    still be ~1e-3 from it).  The trained network's judged start must reach
    the same solutions (within 1e-6, gauge-aligned) in at most half the
    iterations summed over chanblocks."""
    ntiles, nch = 24, 48
    tight = (400, 1e-15)
    X, Y = [], []
    for seed in range(6):
        blocks = ws.DriftSky(ntiles, nch, 2, 3, seed=100 + seed).generate()
        sols, _, _ = solve_sequence(blocks, None, tight)
        for k in range(1, len(sols)):
            X.append(ws.features(sols[k - 1]))
            Y.append(ws.targets(sols[k - 1], sols[k]))
    X, Y = np.concatenate(X), np.concatenate(Y)
    ok = np.isfinite(X).all(axis=1) & np.isfinite(Y).all(axis=1)
    mlp = ws.WarmStartMLP(hidden=128, num_hidden=3, seed=0)
    losses = mlp.train(X[ok], Y[ok], epochs=60, batch=256, lr=1e-3)
    assert losses[-1] < 0.01 * losses[0], losses

    blocks = ws.DriftSky(ntiles, nch, 2, 4, seed=999).generate()
    s_id, it_id, _ = solve_sequence(blocks, None, tight)
    s_ws, it_ws, chose = solve_sequence(blocks, mlp, tight)
    assert np.mean(np.concatenate(chose[1:])) > 0.8
    total_id = sum(int(i.sum()) for i in it_id[1:])
    total_ws = sum(int(i.sum()) for i in it_ws[1:])
    assert 2 * total_ws <= total_id, (total_ws, total_id)
    worst_id = max(int(i.max()) for i in it_id[1:])
    worst_ws = max(int(i.max()) for i in it_ws[1:])
    assert worst_ws < worst_id, (worst_ws, worst_id)
    for k, (data, model, g) in enumerate(blocks[1:], start=1):
        # the solver's fixed point: iterate from the true gains
        d, m = torch.from_numpy(data).cuda(), torch.from_numpy(model).cuda()
        dj = torch.from_numpy(g.copy()).cuda()
        cal.calibrate_timeblock(d, m, dj, (0, data.shape[0]), 60, 1e-30, 1e-4)
        fp = ws.gauge_align(dj.cpu().numpy())
        scale = np.max(np.abs(fp))
        w, i = ws.gauge_align(s_ws[k]), ws.gauge_align(s_id[k])
        assert np.max(np.abs(w - i)) / scale < 1e-6, k
        assert np.max(np.abs(w - fp)) / scale < 1e-6, k
        assert np.max(np.abs(i - fp)) / scale < 1e-6, k


def test_fallback_to_identity_when_proposal_is_worse():
    blocks = ws.DriftSky(12, 8, 2, 1, seed=5).generate()
    data, model, g = blocks[0]
    d, m = torch.from_numpy(data).cuda(), torch.from_numpy(model).cuda()
    rng = np.random.default_rng(0)
    bad = rng.normal(0, 5.0, g.shape)  # a nonsense proposal
    good = g.copy()
    prop = bad.copy()
    prop[:, ::2] = good[:, ::2]  # good on even chanblocks only
    start, use = ws.judge(d, m, (0, data.shape[0]), prop)
    assert use[::2].all() and not use[1::2].any()
    np.testing.assert_array_equal(start[:, 1::2], ws.identity_gains(12, 8)[:, 1::2])


def awkward_solutions(ntiles, nch, seed):
    """Previous solutions with the cases the frames must handle: a NaN
    chanblock, a failed tile, a reference tile with zero XX, tiny YY."""
    rng = np.random.default_rng(seed)
    p = rng.normal(size=(ntiles, nch, 8))
    p[..., 0] += 2.0
    p[..., 6] += 2.0
    p[:, 3, :] = np.nan          # a failed chanblock
    p[5, :, :] = np.nan          # a failed tile
    p[0, 7, 0:2] = 0.0           # reference tile XX zero: no rotation
    p[2, 9, 6:8] = 1e-9          # YY below the frame threshold
    return p


def test_device_features_match_host_restatement():
    p = awkward_solutions(20, 17, 3)
    x = ws.features_device(torch.from_numpy(p).cuda()).cpu().numpy()
    ref = ws.features(p)
    assert x.shape == ref.shape
    np.testing.assert_allclose(x, ref, rtol=2e-6, atol=2e-6)


def test_device_proposal_matches_host_restatement():
    rng = np.random.default_rng(4)
    mlp = ws.WarmStartMLP(hidden=64, num_hidden=3, seed=2)
    q = mlp.get_params()
    mlp.set_params(q + rng.normal(0, 0.02, q.size).astype(np.float32))
    p = awkward_solutions(20, 17, 5)
    d_start, d_use = mlp.propose_device(torch.from_numpy(p).cuda())
    assert d_use is None
    host = mlp.propose(p)
    host = np.where(np.isfinite(host), host, ws.identity_gains(20, 17))
    np.testing.assert_allclose(d_start.cpu().numpy(), host, rtol=1e-5, atol=1e-5)


def test_device_chain_judges_like_the_host():
    """propose_device with the timeblock's data runs the judge: its choice
    and starting gains equal the host-driven judge of the same proposal."""
    blocks = ws.DriftSky(16, 12, 2, 2, seed=8).generate()
    mlp = ws.WarmStartMLP(hidden=32, num_hidden=2, seed=4)
    (data0, model0, _), (data1, model1, _) = blocks
    d0, m0 = torch.from_numpy(data0).cuda(), torch.from_numpy(model0).cuda()
    sol, _, _, _ = ws.calibrate_warm(d0, m0, (0, data0.shape[0]), None, None, max_iterations=100)
    sol_np = sol.cpu().numpy()
    sol_np[:, 4, :] = np.nan  # one failed chanblock: its proposal is the identity
    d1, m1 = torch.from_numpy(data1).cuda(), torch.from_numpy(model1).cuda()
    d_start, d_use = mlp.propose_device(torch.from_numpy(sol_np).cuda(), d1, m1, (0, data1.shape[0]))
    prop, _ = mlp.propose_device(torch.from_numpy(sol_np).cuda())
    start, use = ws.judge(d1, m1, (0, data1.shape[0]), prop.cpu().numpy())
    np.testing.assert_array_equal(d_use.cpu().numpy().astype(bool), use)
    np.testing.assert_array_equal(d_start.cpu().numpy(), start)
    assert use.sum() >= 8  # the previous solution is a far better start than identity on most chanblocks
