"""DI calibration on the GPU against the CPU oracle and the reference's
known-answer tests (di_calibrate/tests.rs).

Solutions are compared within 1e-10 relative (normwise over all tiles and
chanblocks, NaN patterns identical); iteration counts, convergence flags and
failed-tile counts must be equal."""

import numpy as np
import pytest

from mwa_hyperdrive_b200 import synth

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("no CUDA device", allow_module_level=True)

from mwa_hyperdrive_b200 import calibrate as cal  # noqa: E402


def identity(n, nch=1):
    j = np.zeros((n, nch, 8))
    j[..., 0] = 1
    j[..., 6] = 1
    return j


def gpu_timeblock(data, model, dj0, t0, t1, max_iter=50, stop=1e-8, min_thr=1e-4, pols="XX_XY_YX_YY",
                  form="plain"):
    d = torch.from_numpy(np.ascontiguousarray(data, np.float32)).cuda()
    m = torch.from_numpy(np.ascontiguousarray(model, np.float32)).cuda()
    dj = torch.from_numpy(np.ascontiguousarray(dj0, np.float64)).cuda()
    res = cal.calibrate_timeblock(d, m, dj, (t0, t1), max_iter, stop, min_thr, pols, form=form)
    return dj.cpu().numpy(), res


def kat(nt, nch, nbl, val):
    d = np.zeros((nt, nch, nbl, 8), np.float32)
    d[..., 0] = val
    d[..., 6] = val
    return d


def test_calibrate_trivial():
    # di_calibrate/tests.rs:37-93
    dj, res = gpu_timeblock(kat(1, 1, 10, 4.0), kat(1, 1, 10, 1.0), identity(5), 0, 1, 20, 1e-8, 1e-5)
    r = res[0]
    assert r.converged and r.num_iterations == 10 and r.num_failed == 0 and r.max_precision < 1e-13
    np.testing.assert_allclose(dj, identity(5) * 2.0, atol=1e-14, rtol=0)


def test_calibrate_trivial_with_flags():
    # di_calibrate/tests.rs:98-235
    data = kat(1, 2, 10, 1.0)
    data[:, 0] = kat(1, 1, 10, 4.0)[:, 0]
    data[:, 1] = kat(1, 1, 10, 9.0)[:, 0]
    data[0, 0, 0, 0] = data[0, 0, 0, 6] = 9000.0
    model = kat(1, 2, 10, 1.0)
    dj, res = gpu_timeblock(data, model, identity(5, 2), 0, 1, 20, 1e-8, 1e-5)
    assert all(r.converged and r.num_failed == 0 for r in res)
    assert not np.allclose(dj[:, 0], identity(5)[:, 0] * 2.0)
    np.testing.assert_allclose(dj[:, 1], identity(5)[:, 0] * 3.0, atol=1e-15, rtol=0)
    data[0, 0, 0] = 0
    model[0, 0, 0] = 0
    dj, res = gpu_timeblock(data, model, identity(5, 2), 0, 1, 20, 1e-8, 1e-5)
    assert [r.num_iterations for r in res] == [10, 12]
    assert all(r.max_precision < 1e-13 for r in res)
    np.testing.assert_allclose(dj[:, 0], identity(5)[:, 0] * 2.0, atol=1e-14, rtol=0)
    np.testing.assert_allclose(dj[:, 1], identity(5)[:, 0] * 3.0, atol=1e-14, rtol=0)


def test_multiple_timeblocks():
    # di_calibrate/tests.rs:657-704
    out, results = cal.calibrate_timeblocks(kat(3, 1, 10, 4.0), kat(3, 1, 10, 1.0), [(0, 1), (1, 2), (2, 3)], 10,
                                            1e-8, 1e-4)
    np.testing.assert_allclose(out, np.broadcast_to(identity(5) * 2.0, out.shape), atol=1e-14, rtol=0)


def test_chanblocks_without_data():
    # di_calibrate/tests.rs:706-770
    z = np.zeros((3, 1, 10, 8), np.float32)
    out, results = cal.calibrate_timeblocks(z, z, [(0, 3)], 10, 1e-8, 1e-4)
    assert np.all(np.isnan(out)) and all(r.num_iterations == 1 for r in results[0])
    one = kat(3, 1, 10, 1.0)
    out, results = cal.calibrate_timeblocks(one, one, [(0, 3)], 10, 1e-8, 1e-4)
    assert not np.any(np.isnan(out)) and all(r.num_iterations == 1 for r in results[0])


def test_recalibrating_failed_chanblocks():
    # di_calibrate/tests.rs:772-844
    data, model = kat(1, 3, 10, 4.0), kat(1, 3, 10, 1.0)
    dj0 = identity(5, 3)
    dj0[:, 1] = 0
    dj, res = gpu_timeblock(data, model, dj0, 0, 1, 10, 1e-8, 1e-4)
    assert [r.num_iterations for r in res] == [10, 2, 10]
    dj, res = gpu_timeblock(data, model, np.zeros((5, 3, 8)), 0, 1, 10, 1e-8, 1e-4)
    assert not any(r.converged for r in res)


def compare(oracle, data, model, dj0, t0, t1, max_iter=50, stop=1e-8, min_thr=1e-4, pols="XX_XY_YX_YY"):
    code = {"XX_XY_YX_YY": 0, "XX": 1, "YY": 2, "XX_YY": 3, "XX_YY_XY": 4}[pols]
    dj_g, res_g = gpu_timeblock(data, model, dj0, t0, t1, max_iter, stop, min_thr, pols)
    dj_o, res_o = oracle.calibrate_timeblock(data, model, dj0, t0, t1, max_iter, stop, min_thr, code)
    assert [r.num_iterations for r in res_g] == [r["num_iterations"] for r in res_o]
    assert [r.converged for r in res_g] == [r["converged"] for r in res_o]
    assert [r.num_failed for r in res_g] == [r["num_failed"] for r in res_o]
    np.testing.assert_array_equal(np.isnan(dj_g), np.isnan(dj_o))
    ok = ~np.isnan(dj_o)
    if ok.any():
        err = np.linalg.norm(dj_g[ok] - dj_o[ok]) / np.linalg.norm(dj_o[ok])
        assert err < 1e-10, err
    for rg, ro in zip(res_g, res_o):
        if np.isfinite(ro["max_precision"]) and ro["max_precision"] > 0:
            assert abs(rg.max_precision - ro["max_precision"]) <= 1e-6 * abs(ro["max_precision"]) + 1e-30
    return dj_g, res_g


@pytest.mark.parametrize("ntiles,nt,nch,snr", [(8, 2, 5, None), (20, 4, 6, 10.0), (37, 3, 4, 30.0)])
def test_random_problems_match_oracle(oracle, ntiles, nt, nch, snr):
    rng = np.random.default_rng(ntiles)
    nbl = ntiles * (ntiles - 1) // 2
    model = synth.random_model(nt, nch, nbl, rng)
    g = synth.truth_gains(ntiles, nch, rng)
    data = synth.corrupt(model, g, rng, snr)
    compare(oracle, data, model, identity(ntiles, nch), 0, nt)


def test_128_tiles_noisy(oracle):
    rng = np.random.default_rng(128)
    ntiles, nt, nch = 128, 2, 3
    nbl = ntiles * (ntiles - 1) // 2
    model = synth.random_model(nt, nch, nbl, rng)
    data = synth.corrupt(model, synth.truth_gains(ntiles, nch, rng), rng, 10.0)
    dj, res = compare(oracle, data, model, identity(ntiles, nch), 0, nt)
    assert all(r.converged for r in res)


@pytest.mark.parametrize("pols", ["XX", "YY", "XX_YY"])
def test_single_pol_division(oracle, pols):
    rng = np.random.default_rng(7)
    ntiles, nt, nch = 12, 2, 3
    nbl = ntiles * (ntiles - 1) // 2
    model = synth.random_model(nt, nch, nbl, rng)
    data = synth.corrupt(model, synth.truth_gains(ntiles, nch, rng, leak_sigma=0.0), rng, None)
    if pols == "XX":
        model[..., 2:] = 0
        data[..., 2:] = 0
    elif pols == "YY":
        model[..., :6] = 0
        data[..., :6] = 0
    compare(oracle, data, model, identity(ntiles, nch), 0, nt, pols=pols)


def test_failed_chanblock_retry_and_flagged_tile(oracle):
    rng = np.random.default_rng(11)
    ntiles, nt, nch = 10, 2, 7
    nbl = ntiles * (ntiles - 1) // 2
    model = synth.random_model(nt, nch, nbl, rng)
    data = synth.corrupt(model, synth.truth_gains(ntiles, nch, rng), rng, 20.0)
    # chanblock 3 has no data -> fails on iteration 1, then stays failed;
    # chanblock 5 starts from zero gains and fails, then is retried
    data[:, 3] = 0
    model[:, 3] = 0
    dj0 = identity(ntiles, nch)
    dj0[:, 5] = 0
    # a flagged tile: all its baselines zero in chanblock 1
    i, j = np.triu_indices(ntiles, 1)
    sel = (i == 4) | (j == 4)
    data[:, 1, sel] = 0
    model[:, 1, sel] = 0
    compare(oracle, data, model, dj0, 0, nt, max_iter=30)


def compare_collapsed(oracle, data, model, dj0, t0, t1, form, max_iter=50, stop=1e-8, min_thr=1e-4):
    """The collapsed forms regroup the timestep sums (FP64: same iteration
    counts, solutions to rounding; FP32 covariances: solutions to ~1e-7)."""
    dj_g, res_g = gpu_timeblock(data, model, dj0, t0, t1, max_iter, stop, min_thr, form=form)
    dj_o, res_o = oracle.calibrate_timeblock(data, model, dj0, t0, t1, max_iter, stop, min_thr, 0)
    assert [r.converged for r in res_g] == [r["converged"] for r in res_o]
    it_g = np.array([r.num_iterations for r in res_g])
    it_o = np.array([r["num_iterations"] for r in res_o])
    if form == "collapsed":
        np.testing.assert_array_equal(it_g, it_o)
    else:
        assert np.max(np.abs(it_g - it_o)) <= 2, (it_g, it_o)
    np.testing.assert_array_equal(np.isnan(dj_g), np.isnan(dj_o))
    ok = ~np.isnan(dj_o)
    err = np.linalg.norm(dj_g[ok] - dj_o[ok]) / np.linalg.norm(dj_o[ok]) if ok.any() else 0.0
    return err


# tile counts: one block (8), an odd number of blocks (20: 3), 128 (36 blocks,
# a 3-slot shared-memory ring in the FP32 form), and above 155 tiles, where
# the FP32 form's ring is 2 slots deep (200: 91 blocks; 256, the largest
# array the kernel takes: 136 blocks)
@pytest.mark.parametrize("form,tol", [("collapsed", 1e-9), ("collapsed_f32", 1e-6)])
@pytest.mark.parametrize("ntiles,nt,nch,snr", [(8, 2, 5, None), (20, 4, 6, 10.0), (128, 14, 3, 10.0),
                                               (200, 2, 2, 10.0), (256, 2, 2, 10.0)])
def test_collapsed_forms_match_oracle(oracle, form, tol, ntiles, nt, nch, snr):
    rng = np.random.default_rng(ntiles + nt)
    nbl = ntiles * (ntiles - 1) // 2
    model = synth.random_model(nt, nch, nbl, rng)
    g = synth.truth_gains(ntiles, nch, rng)
    data = synth.corrupt(model, g, rng, snr)
    err = compare_collapsed(oracle, data, model, identity(ntiles, nch), 0, nt, form)
    assert err < tol, err


@pytest.mark.parametrize("form", ["collapsed", "collapsed_f32"])
def test_collapsed_forms_retry_and_timeblock_offset(oracle, form):
    rng = np.random.default_rng(11)
    ntiles, nt, nch = 10, 4, 7
    nbl = ntiles * (ntiles - 1) // 2
    model = synth.random_model(nt, nch, nbl, rng)
    data = synth.corrupt(model, synth.truth_gains(ntiles, nch, rng), rng, 20.0)
    data[:, 3] = 0
    model[:, 3] = 0
    dj0 = identity(ntiles, nch)
    dj0[:, 5] = 0
    err = compare_collapsed(oracle, data, model, dj0, 1, 3, form, max_iter=30)
    assert err < (1e-9 if form == "collapsed" else 1e-6), err


@pytest.mark.parametrize("form", ["plain", "collapsed", "collapsed_f32"])
def test_timeblocks_graph_equals_per_timeblock_calls(form):
    """calibrate_timeblocks runs every timeblock's first pass as one CUDA
    graph and the retry of failed chanblocks afterwards; its solutions and
    results equal those of one hdc_calibrate_timeblock call per timeblock,
    including a chanblock that fails (zero data) and is retried from its
    neighbours: bit for bit for the collapsed forms (deterministic block
    reductions); to rounding for the plain form, whose shared-memory FP64
    atomics add in a run-dependent order."""
    rng = np.random.default_rng(21)
    ntiles, nt, nch = 12, 6, 9
    nbl = ntiles * (ntiles - 1) // 2
    model = synth.random_model(nt, nch, nbl, rng)
    data = synth.corrupt(model, synth.truth_gains(ntiles, nch, rng), rng, 30.0)
    data[:, 3] = 0
    model[:, 3] = 0
    tbs = [(0, 2), (2, 5), (5, 6)]
    out, results = cal.calibrate_timeblocks(data, model, tbs, 40, 1e-8, 1e-4, form=form)
    d, m = torch.from_numpy(data).cuda(), torch.from_numpy(model).cuda()
    for k, tb in enumerate(tbs):
        dj = torch.from_numpy(identity(ntiles, nch)).cuda()
        res = cal.calibrate_timeblock(d, m, dj, tb, 40, 1e-8, 1e-4, form=form)
        if form == "plain":
            np.testing.assert_allclose(out[k], dj.cpu().numpy(), rtol=1e-10, atol=1e-12)
        else:
            np.testing.assert_array_equal(out[k], dj.cpu().numpy())
        assert [r.num_iterations for r in results[k]] == [r.num_iterations for r in res]
        assert [r.converged for r in results[k]] == [r.converged for r in res]
        assert not res[3].converged and sum(r.converged for r in res) >= nch - 2


def test_calibrate_chanblocks_one_pass_and_listed(oracle):
    """hdc_calibrate_chanblocks: one pass without the retry gives the
    oracle's per-chanblock solves; a list re-runs only the named chanblocks
    (the building block of the chanblock-sharded calibration)."""
    import ctypes

    from mwa_hyperdrive_b200 import _lib

    rng = np.random.default_rng(21)
    ntiles, nt, nch = 12, 2, 5
    nbl = ntiles * (ntiles - 1) // 2
    model = synth.random_model(nt, nch, nbl, rng)
    data = synth.corrupt(model, synth.truth_gains(ntiles, nch, rng), rng, 30.0)
    start = identity(ntiles, nch)
    start[:, 2] = 0.0  # fails without the retry
    d, m = torch.from_numpy(data).cuda(), torch.from_numpy(model).cuda()
    dj = torch.from_numpy(start.copy()).cuda()
    res = (_lib.HdcCalResult * nch)()
    _lib.check(_lib.lib().hdc_calibrate_chanblocks(d.data_ptr(), m.data_ptr(), nt, 0, nt, nch, nbl, dj.data_ptr(), 50,
                                                   1e-8, 1e-4, 0, None, 0, res, 0, None), "hdc_calibrate_chanblocks")
    got = dj.cpu().numpy()
    for c in range(nch):
        ref, r = oracle.calibrate(data, model, c, start[:, c], 50, 1e-8, 1e-4, 0)
        assert res[c].num_iterations == r.num_iterations and bool(res[c].converged) == bool(r.converged)
        np.testing.assert_array_equal(np.isnan(got[:, c]), np.isnan(ref))
    assert not res[2].converged
    # re-run chanblock 2 alone from its neighbours' mean: it converges, the others are untouched
    before = got.copy()
    seedv = 0.5 * (got[:, 1] + got[:, 3])
    dj[:, 2] = torch.from_numpy(seedv).cuda()
    lst = (ctypes.c_int * 1)(2)
    _lib.check(_lib.lib().hdc_calibrate_chanblocks(d.data_ptr(), m.data_ptr(), nt, 0, nt, nch, nbl, dj.data_ptr(), 50,
                                                   1e-8, 1e-4, 0, lst, 1, res, 0, None), "hdc_calibrate_chanblocks")
    after = dj.cpu().numpy()
    assert res[2].converged
    np.testing.assert_array_equal(after[:, [0, 1, 3, 4]], before[:, [0, 1, 3, 4]])
    ref, r = oracle.calibrate(data, model, 2, seedv, 50, 1e-8, 1e-4, 0)
    assert res[2].num_iterations == r.num_iterations
    assert np.max(np.abs(after[:, 2] - ref)) < 1e-10


def test_sharded_calibration_with_the_gpu_solver(oracle, tmp_path):
    """shard.calibrate_timeblock_sharded with the GPU chanblock solver on one
    rank equals calibrate_timeblock (first pass and band-wide retry)."""
    import torch.distributed as dist

    from mwa_hyperdrive_b200 import shard

    rng = np.random.default_rng(22)
    ntiles, nt, nch = 12, 2, 6
    nbl = ntiles * (ntiles - 1) // 2
    model = synth.random_model(nt, nch, nbl, rng)
    data = synth.corrupt(model, synth.truth_gains(ntiles, nch, rng), rng, 30.0)
    start = identity(ntiles, nch)
    start[:, 2] = start[:, 3] = 0.0
    d, m = torch.from_numpy(data).cuda(), torch.from_numpy(model).cuda()
    ref_dj, ref_res = gpu_timeblock(data, model, start, 0, nt, form="collapsed_f32")
    dist.init_process_group("gloo", init_method=f"file://{tmp_path}/pg", rank=0, world_size=1)
    try:
        solver = shard.gpu_chanblock_solver(d, m, (0, nt), form="collapsed_f32")
        sols, res = shard.calibrate_timeblock_sharded(solver, start.copy(), 0, nch)
    finally:
        dist.destroy_process_group()
    np.testing.assert_array_equal(np.isnan(sols), np.isnan(ref_dj))
    ok = ~np.isnan(ref_dj)
    assert np.max(np.abs(sols[ok] - ref_dj[ok])) == 0.0
    assert [r["num_iterations"] for r in res] == [r.num_iterations for r in ref_res]
