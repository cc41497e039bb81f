"""Differentiation check: the autograd wrapper's backward (the library's
gradient kernels, partial-derivative convention) against central finite
differences in FP64, and in FP32 against the reference's evaluate_cpu
gradient (tied convention) after symmetrising."""
import os

import numpy as np
import pytest

from ccmpred_b200 import Evaluator, nsingle_padded, synth

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def test_pack_unpack_roundtrip():
    import torch
    from ccmpred_b200.autograd import pack, unpack
    L = 7
    x = torch.from_numpy(synth.random_x(L, 3, symmetric=False)).double()
    V, W = unpack(x, L)
    assert torch.equal(pack(V, W), x)


def test_gradcheck_small_fp64(gpu):
    """torch.autograd.gradcheck over every entry of V and W (L=4, N=12)."""
    import torch
    from ccmpred_b200.autograd import pseudo_likelihood, unpack
    msa = synth.generate(synth.MSAConfig("ag", 4, 12, seed=81))
    ev = Evaluator(msa, path="simt_f64", gradient="partial", lambda_pair=0.6)
    x = torch.from_numpy(synth.random_x(4, 82, w_sd=0.3, symmetric=False)).double().cuda()
    V, W = unpack(x, 4)
    V = V.clone().requires_grad_(True)
    W = W.clone().requires_grad_(True)
    assert torch.autograd.gradcheck(lambda v, w: pseudo_likelihood(v, w, ev), (V, W),
                                    eps=1e-6, atol=1e-6, rtol=1e-5)
    ev.close()


def test_central_differences_500_coordinates_fp64(gpu):
    """L=150, N=2000: analytic gradient vs (f(x+h e_i) - f(x-h e_i)) / 2h, h = 1e-4,
    on 500 random coordinates of V and W (self blocks and padding included)."""
    import torch
    cfg = synth.AUTOGRAD_150x2000
    msa = synth.generate(cfg)
    L = cfg.ncol
    ev = Evaluator(msa, path="simt_f64", gradient="partial")
    x = torch.from_numpy(synth.random_x(L, 83, symmetric=False)).double().cuda()
    g = torch.empty_like(x)
    ev.evaluate(x, g)
    rng = np.random.default_rng(84)
    nsp = nsingle_padded(L)
    idx = np.concatenate([rng.integers(0, 20 * L, 100), rng.integers(nsp, x.numel(), 400)])
    h = 1e-4
    gfd = np.empty(len(idx))
    scratch = torch.empty_like(x)
    for t, i in enumerate(idx):
        x[i] += h
        fp = ev.evaluate(x, scratch)
        x[i] -= 2 * h
        fm = ev.evaluate(x, scratch)
        x[i] += h
        gfd[t] = (fp - fm) / (2 * h)
    ga = g.cpu().numpy()[idx]
    err = np.abs(ga - gfd)
    assert np.all(err <= 1e-4 * np.maximum(1.0, np.abs(ga))), err.max()
    ev.close()


@pytest.mark.parametrize("path", ["tc_i8x3", "tc_i8sp", "tc_bf16x2", "simt_f32"])
def test_partial_symmetrised_matches_reference_fp32(gpu, path):
    """FP32: partial + partial^T (k != j) equals the reference's evaluate_cpu
    gradient (golden vector, symmetric x)."""
    import torch
    from ccmpred_b200.autograd import pseudo_likelihood, unpack
    d = np.load(os.path.join(GOLDEN, "eval_L14_N45_rand.npz"))
    msa, x0, w = d["msa"], d["x"], d["weights"]
    L = msa.shape[1]
    ev = Evaluator(msa, weights=w, lambda_single=float(d["lambda_single"]),
                   lambda_pair=float(d["lambda_pair"]), path=path, gradient="partial")
    V, W = unpack(torch.from_numpy(x0).cuda(), L)
    V = V.clone().requires_grad_(True)
    W = W.clone().requires_grad_(True)
    f = pseudo_likelihood(V, W, ev)
    f.backward()
    assert abs(f.item() - float(d["f"])) / abs(float(d["f"])) < 2e-6
    gV = V.grad.cpu().numpy().astype(np.float64)             # [j, a]
    gW = W.grad.cpu().numpy().astype(np.float64)             # [k, j, b, a]
    tied = gW + gW.transpose(1, 0, 3, 2)
    idx = np.arange(L)
    tied[idx, idx] = 0.0
    nsp = nsingle_padded(L)
    ref = d["g"].astype(np.float64)
    refV = ref[: 20 * L].reshape(20, L).T
    refW = ref[nsp:].reshape(21, L, 32, L)[:, :, :21, :].transpose(1, 3, 0, 2)
    # self blocks of the reference g are 2 lambda2 W (zero here: admissible x)
    scale = np.linalg.norm(ref)
    assert np.linalg.norm(gV - refV) / scale < 1e-5
    assert np.linalg.norm(tied - refW) / scale < 1e-5
    ev.close()
