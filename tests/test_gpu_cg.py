"""Device conjugate gradient (ccm_conjugrad_gpu) vs an FP64 host CG with the
same rules (oracle_conjugrad_f64).  libconjugrad is absent from the reference,
so trajectory parity with the reference optimizer is not pinned; these tests
check the device loop against its own specification."""
import numpy as np
import pytest

from ccmpred_b200 import Evaluator, _lib, synth
from ccmpred_b200.host import init_bias

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("path", ["tc_i8x3", "tc_i8sp", "tc_bf16x2", "simt_f32"])
def test_cg_matches_fp64_host_cg(gpu, oracle_mod, path):
    import torch
    msa = synth.generate(synth.MSAConfig("cg", 24, 300, n_pairs=4, dup_frac=0.2, seed=61))
    N, L = msa.shape
    w = oracle_mod.oracle_weights(msa, 0.8)
    lam1, lam2 = 0.01, 0.2 * (L - 1)
    x0 = init_bias(msa)
    iters = 12
    xh, fh, it_h, ev_h, st_h = oracle_mod.oracle_conjugrad(msa, w, lam1, lam2, x0,
                                                          max_iter=iters, eps=0.0)
    ev = Evaluator(msa, weights=w, lambda_single=lam1, lambda_pair=lam2, path=path)
    xd = torch.from_numpy(x0.copy()).cuda()
    seen = []
    res = ev.minimize(xd, max_iterations=iters, epsilon=0.0,
                      progress=lambda k, ls, fx, xn, gn, st: seen.append((k, ls, fx)) and False)
    ev.close()
    assert res.status == _lib.CG_ERR_MAXITER and st_h == -1023
    assert res.iterations == it_h == iters
    assert [k for k, _, _ in seen] == list(range(1, iters + 1))
    fd = np.array([fx for _, _, fx in seen])
    assert np.all(np.diff(fd) < 0)                      # monotone decrease
    assert np.allclose(fd, fh[1:], rtol=2e-5)            # same trajectory as FP64
    assert abs(res.fx - fh[-1]) / abs(fh[-1]) < 2e-5
    xg = xd.cpu().numpy().astype(np.float64)
    assert np.linalg.norm(xg - xh) / np.linalg.norm(xh) < 1e-3


def test_cg_converges_and_recovers_planted_contacts(gpu):
    import torch
    from ccmpred_b200.host import contact_map
    cfg = synth.MSAConfig("cg2", 40, 2000, n_pairs=8, seed=62)
    msa = synth.generate(cfg)
    N, L = msa.shape
    from ccmpred_b200 import calculate_weights
    w = calculate_weights(msa, 0.8)
    ev = Evaluator(msa, weights=w)
    xd = torch.from_numpy(init_bias(msa)).cuda()
    res = ev.minimize(xd, max_iterations=200)
    ev.close()
    assert res.status == _lib.CG_SUCCESS and res.iterations < 200
    cmap, _ = contact_map(xd.cpu().numpy(), L, apc=True)
    # the planted pairs are the strongest contacts
    rng = np.random.Generator(np.random.PCG64(cfg.seed))
    iu = np.triu_indices(L, 1)
    order = np.argsort(-cmap[iu])
    top = {(int(iu[0][i]), int(iu[1][i])) for i in order[:8]}
    planted = planted_pairs(cfg)
    assert len(top & planted) >= 6, (top, planted)


def planted_pairs(cfg):
    """Re-derive the planted column pairs of synth.generate (same RNG stream)."""
    from ccmpred_b200.synth import Q
    rng = np.random.Generator(np.random.PCG64(cfg.seed))
    L, N = cfg.ncol, cfg.nrow
    rng.dirichlet(np.full(Q - 1, 0.5), size=L)
    rng.random((N, L))
    rng.random((N, L))
    npairs = min(cfg.n_pairs, L // 2)
    cols = rng.permutation(L)[: 2 * npairs].reshape(npairs, 2)
    return {(int(min(a, b)), int(max(a, b))) for a, b in cols}


@pytest.mark.parametrize("path", ["tc_i8x3", "tc_i8sp", "tc_bf16x2", "tc_bf16x3", "simt_f32"])
def test_cg_result_is_the_evaluation_at_the_returned_x(gpu, path):
    """On the tensor-core paths each trial's step x_t = x + alpha s is fused into the
    first pass over x (tc_prep; the column-max pass of the integer path), which
    writes x_t and evaluates it.  The x that the
    CG returns is such an x_t: evaluating it again must give the CG's f exactly,
    and the gradient left in the CG's last accepted trial is that of this x."""
    import torch
    msa = synth.generate(synth.MSAConfig("cgstep", 53, 700, n_pairs=5, seed=63))
    ev = Evaluator(msa, path=path)
    for iters in (1, 7):
        xd = torch.from_numpy(init_bias(msa)).cuda()
        res = ev.minimize(xd, max_iterations=iters, epsilon=0.0)
        g = torch.empty_like(xd)
        f = ev.evaluate(xd, g)
        assert f == res.fx
        assert abs(float(torch.linalg.vector_norm(g.double())) - res.gnorm) <= 1e-12 * res.gnorm
    ev.close()


@pytest.mark.parametrize("path", ["tc_i8sp", "tc_bf16x2", "simt_f32"])
def test_whole_solve_graph_equals_per_iteration_loop(gpu, oracle_mod, path):
    """Without a progress callback the whole solve is one graph launch (line
    search, direction update and stopping test on the device, in conditional
    nodes); with one, the host launches one line-search graph per iteration.
    Both apply the same kernels and rules: the same x bit for bit, the same
    iterations and evaluations, and the trajectory of the FP64 restatement."""
    import torch
    msa = synth.generate(synth.MSAConfig("cgw", 30, 400, n_pairs=4, dup_frac=0.2, seed=64))
    N, L = msa.shape
    w = oracle_mod.oracle_weights(msa, 0.8)
    lam1, lam2 = 0.01, 0.2 * (L - 1)
    x0 = init_bias(msa)
    ev = Evaluator(msa, weights=w, lambda_single=lam1, lambda_pair=lam2, path=path)
    xa = torch.from_numpy(x0.copy()).cuda()
    ra = ev.minimize(xa, max_iterations=40, epsilon=1e-3)
    xb = torch.from_numpy(x0.copy()).cuda()
    seen = []
    rb = ev.minimize(xb, max_iterations=40, epsilon=1e-3,
                     progress=lambda k, ls, fx, xn, gn, st: seen.append(k) and False)
    ev.close()
    assert torch.equal(xa, xb)
    assert (ra.status, ra.iterations, ra.evaluations, ra.fx) == \
        (rb.status, rb.iterations, rb.evaluations, rb.fx)
    assert seen == list(range(1, rb.iterations + 1))
    _, fh, it_h, ev_h, st_h = oracle_mod.oracle_conjugrad(msa, w, lam1, lam2, x0.astype(np.float64),
                                                          max_iter=40, eps=1e-3)
    assert ra.status == st_h and ra.iterations == it_h and ra.evaluations == ev_h
    assert abs(ra.fx - fh[-1]) / abs(fh[-1]) < 2e-5


@pytest.mark.parametrize("path", ["tc_i8sp", "tc_i8x3"])
@pytest.mark.parametrize("whole_solve", [True, False])
def test_padding_free_passes(gpu, path, whole_solve):
    """x0 with zero padding states: the solve keeps them exactly zero and its vector
    passes skip them; the trajectory equals that of a solve visiting every element
    (up to the summation order of the FP64 dots).  x0 with a nonzero padding state:
    the check sees it and the solve visits every element, bit for bit as when
    skipping is forbidden.  whole_solve=False: the per-iteration graphs (a progress
    callback)."""
    import torch
    from ccmpred_b200 import lib, nsingle_padded
    msa = synth.generate(synth.MSAConfig("pad", 37, 500, n_pairs=3, seed=67))
    L = msa.shape[1]
    nsp = nsingle_padded(L)
    progress = None if whole_solve else (lambda *a: False)

    def solve(x0, allow):
        with Evaluator(msa, path=path) as ev:
            assert lib().ccm_debug_set_cg_skip_padding(ev.handle, allow) == 0
            xd = torch.from_numpy(x0.copy()).cuda()
            res = ev.minimize(xd, max_iterations=10, epsilon=0.0, progress=progress)
            return res, xd.cpu().numpy()

    x0 = init_bias(msa)
    r1, x1 = solve(x0, 1)
    r0, xz = solve(x0, 0)
    assert r1.iterations == r0.iterations == 10 and r1.evaluations == r0.evaluations
    assert abs(r1.fx - r0.fx) <= 1e-9 * abs(r0.fx)
    np.testing.assert_allclose(x1, xz, rtol=0, atol=1e-6)
    pad = x1[nsp:].reshape(21, L, 32, L)[:, :, 21:, :]
    assert not np.any(pad.view(np.uint32))                 # still exactly +0.0
    xp = x0.copy()
    xp[nsp:].reshape(21, L, 32, L)[3, 5, 25, 7] = 1e-3      # one nonzero padding state
    rp1, xp1 = solve(xp, 1)
    rp0, xp0 = solve(xp, 0)
    assert rp1.fx == rp0.fx and np.array_equal(xp1.view(np.uint32), xp0.view(np.uint32))
