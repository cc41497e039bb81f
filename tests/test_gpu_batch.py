"""Batched solves (ccm_solve_batch): every alignment's result equals that of a
standalone solve of the same alignment (contexts are independent and each
solve is deterministic), whatever the number of concurrent workers and the
share of SMs each worker's contexts may use."""
import numpy as np
import pytest

from ccmpred_b200 import _lib, solve_batch, synth

pytestmark = pytest.mark.gpu


def test_batch_matches_standalone_solves(gpu):
    """The wave solver (all solves of a wave in one graph launch; several waves
    here) and the host-thread solver (4 workers, and 1) give every alignment the
    same result: the same kernels and rules run per alignment either way."""
    msas = synth.batch_workload(10, seed0=500)
    msas = [m[: min(len(m), 1500)] for m in msas]          # keep the test short
    resw, mapsw = solve_batch(msas, max_iterations=40, waves=True, wave_max=4)
    res4, maps4 = solve_batch(msas, workers=4, max_iterations=40, waves=False)
    res1, maps1 = solve_batch(msas, workers=1, max_iterations=40, waves=False)
    for rw, r4, r1, mw, m4, m1 in zip(resw, res4, res1, mapsw, maps4, maps1):
        assert rw.status in (_lib.CG_SUCCESS, _lib.CG_ERR_MAXITER)
        assert rw.iterations == r4.iterations == r1.iterations
        assert rw.evaluations == r4.evaluations and rw.fx == r4.fx == r1.fx
        assert np.array_equal(mw, m4) and np.array_equal(m4, m1)
        assert np.all(np.isfinite(mw))


@pytest.mark.parametrize("gradient", ["tied", "partial"])
def test_sm_share_gives_identical_results(gpu, gradient):
    """max_sms only changes which CTA pair runs which tile: every tile is computed
    the same way, the loss partials are summed in a fixed order and every gradient
    element receives exactly one add, so f and g are bit-for-bit the same."""
    import torch
    from ccmpred_b200 import Evaluator
    msa = synth.generate(synth.MSAConfig("share", 150, 1400, n_pairs=10, seed=71))
    x = torch.from_numpy(synth.random_x(150, 72, symmetric=(gradient == "tied"))).cuda()
    out = []
    for max_sms in (0, 30, 8, 2):
        ev = Evaluator(msa, gradient=gradient, max_sms=max_sms)
        g = torch.empty_like(x)
        f = ev.evaluate(x, g)
        out.append((f, g.cpu().numpy()))
        ev.close()
    for f, g in out[1:]:
        assert f == out[0][0]
        assert np.array_equal(g, out[0][1])


def test_batch_with_explicit_share(gpu):
    msas = [m[:800] for m in synth.batch_workload(4, seed0=600)]
    ra, ma = solve_batch(msas, workers=2, max_iterations=15, sms_per_worker=12, waves=False)
    rb, mb = solve_batch(msas, workers=2, max_iterations=15, sms_per_worker=-1, waves=False)
    for a, b, x, y in zip(ra, rb, ma, mb):
        assert a.iterations == b.iterations and a.fx == b.fx
        assert np.array_equal(x, y)


def test_device_contact_scores_match_host(gpu):
    """ccm_sum_submatrices_gpu reproduces the host sum_submatrices (the reference's
    order of float operations) bit for bit."""
    import torch
    from ccmpred_b200 import host
    from ccmpred_b200._lib import lib
    for L, seed in ((7, 1), (37, 2), (130, 3)):
        x = synth.random_x(L, seed, v_sd=0.3, w_sd=0.2, symmetric=(seed != 2))
        want, _ = host.contact_map(x, L, apc=False)
        xd = torch.from_numpy(x).cuda()
        out = torch.empty(L * L, dtype=torch.float32, device="cuda")
        assert lib().ccm_sum_submatrices_gpu(xd.data_ptr(), out.data_ptr(), L, None) == 0
        torch.cuda.synchronize()
        assert np.array_equal(out.cpu().numpy().reshape(L, L), want)


def test_batch_map_equals_standalone_pipeline(gpu):
    """The batch keeps x on the device and computes the contact map there; the map
    equals that of the host pipeline: weights, init_bias, the device CG, then the
    host sum_submatrices and APC."""
    import torch
    from ccmpred_b200 import Evaluator, calculate_weights, host
    msa = synth.generate(synth.MSAConfig("pipe", 90, 700, n_pairs=9, seed=77))
    res, maps = solve_batch([msa], workers=1, max_iterations=25, epsilon=1e-3)
    w = calculate_weights(msa, 0.8)
    ev = Evaluator(msa, weights=w)
    x = torch.from_numpy(host.init_bias(msa)).cuda()
    r = ev.minimize(x, max_iterations=25, epsilon=1e-3)
    ev.close()
    want, _ = host.contact_map(x.cpu().numpy(), 90, apc=True)
    assert res[0].iterations == r.iterations and res[0].fx == r.fx
    assert np.array_equal(maps[0], want)


def test_batch_rejects_bad_input(gpu):
    with pytest.raises(_lib.CcmError):
        solve_batch([np.zeros((5, 0), dtype=np.uint8)])
