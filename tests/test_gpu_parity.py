"""Parity of the CUDA paths with the oracle (FP64 restatement of
src/evaluate_cpu.c) and with the reference's FP32 results (golden vectors),
through the C ABI.  Tolerances are stated per path and per result:
relative L2 error of f, of the single-field gradient g1 and of the coupling
gradient g2 against the FP64 oracle at identical x."""
import ctypes
import glob
import os

import numpy as np
import pytest

from ccmpred_b200 import Evaluator, _lib, calculate_weights, lib, nsingle_padded, synth

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")

# Error bounds vs the FP64 oracle at identical x, per result:
#   f      relative error of f;
#   g      relative L2 error of the whole gradient (the headline bound, 1e-5);
#   g1, g2 L2 error of the single-field / coupling part divided by the L2 norm
#          of the whole gradient.  At x0 = init_bias the single-field gradient
#          nearly cancels (sum_n w P ~ sum_n w onehot), so its error relative
#          to its own norm is large for every FP32 evaluator, the reference's
#          evaluate_cpu included (1.2e-3 at L=300, N=5000).
TOL = {
    "simt_f32": dict(f=1e-6, g=1e-5, g1=1e-5, g2=1e-5),
    "tc_bf16x2": dict(f=1e-6, g=1e-5, g1=1e-5, g2=1e-5),
    "tc_bf16x3": dict(f=1e-6, g=1e-5, g1=1e-5, g2=1e-5),
    "tc_i8x3": dict(f=1e-6, g=1e-5, g1=1e-5, g2=1e-5),
    "tc_i8sp": dict(f=1e-6, g=1e-5, g1=1e-5, g2=1e-5),
}
PATHS = list(TOL)


def errors(f, g, f64, g64, L):
    nsp = nsingle_padded(L)
    ns = 20 * L
    d = g.astype(np.float64) - g64
    gn = max(np.linalg.norm(g64), 1e-300)
    return dict(f=abs(f - f64) / abs(f64), g=float(np.linalg.norm(d) / gn),
                g1=float(np.linalg.norm(d[:ns]) / gn), g2=float(np.linalg.norm(d[nsp:]) / gn))


def within(e, tol, slack=0.0):
    return all(e[k] < tol[k] + slack for k in tol)


def run(path, msa, w, x, lam1, lam2):
    import torch
    ev = Evaluator(msa, weights=w, lambda_single=lam1, lambda_pair=lam2, path=path)
    xd = torch.from_numpy(np.ascontiguousarray(x, dtype=np.float32)).cuda()
    gd = torch.full_like(xd, float("nan"))
    f = ev.evaluate(xd, gd)
    g = gd.cpu().numpy()
    ev.close()
    return f, g


@pytest.mark.parametrize("path", PATHS)
@pytest.mark.parametrize("fixture", sorted(glob.glob(os.path.join(GOLDEN, "eval_*.npz"))))
def test_golden(gpu, oracle_mod, path, fixture):
    d = np.load(fixture)
    msa, x, w = d["msa"], d["x"], d["weights"]
    lam1, lam2 = float(d["lambda_single"]), float(d["lambda_pair"])
    f, g = run(path, msa, w, x, lam1, lam2)
    assert np.all(np.isfinite(g))
    f64, g64 = oracle_mod.oracle_evaluate(msa, w, lam1, lam2, x)
    e = errors(f, g, f64, g64, msa.shape[1])
    assert within(e, TOL[path]), e
    # against the reference's own FP32 output (its error vs FP64 is ~1e-6 here)
    e_ref = errors(f, g, float(d["f"]), d["g"].astype(np.float64), msa.shape[1])
    assert within(e_ref, TOL[path], slack=2e-6), e_ref


CASES = [
    ("L75_N1000_bias", synth.SMALL_75x1000, "bias"),
    ("L75_N1000_rand", synth.SMALL_75x1000, "rand"),
    ("L13_N64_rand", synth.MSAConfig("t", 13, 64, n_pairs=3, seed=13), "rand"),
    ("L1_N9_rand", synth.MSAConfig("t", 1, 9, seed=14), "rand"),
    ("L7_N1_rand", synth.MSAConfig("t", 7, 1, seed=15), "rand"),
    ("L2_N2_bias", synth.MSAConfig("t", 2, 2, seed=16), "bias"),
    ("L150_N2000_rand", synth.AUTOGRAD_150x2000, "rand"),
]


@pytest.mark.parametrize("path", PATHS)
@pytest.mark.parametrize("name,cfg,xkind", CASES, ids=[c[0] for c in CASES])
def test_synthetic(gpu, oracle_mod, path, name, cfg, xkind):
    msa = synth.generate(cfg)
    N, L = msa.shape
    w = oracle_mod.oracle_weights(msa, 0.8)
    lam1, lam2 = 0.01, 0.2 * max(L - 1, 1)
    if xkind == "bias":
        from ccmpred_b200.host import init_bias
        x = init_bias(msa)
    else:
        x = synth.random_x(L, cfg.seed + 7)
    f, g = run(path, msa, w, x, lam1, lam2)
    f64, g64 = oracle_mod.oracle_evaluate(msa, w, lam1, lam2, x)
    e = errors(f, g, f64, g64, L)
    assert within(e, TOL[path]), e


@pytest.mark.parametrize("path", PATHS)
@pytest.mark.parametrize("kind", ["all_gap", "conserved", "one_state_per_row"])
def test_degenerate_alignments(gpu, oracle_mod, path, kind):
    """Alignments the generator does not produce: every state a gap, every
    column conserved (one state throughout, so P is near one-hot and R small), and
    every row a single repeated state (one-hot slots of one state only)."""
    L, N = 20, 60
    rng = np.random.default_rng(17)
    if kind == "all_gap":
        msa = np.full((N, L), 20, np.uint8)
    elif kind == "conserved":
        msa = np.tile(rng.integers(0, 21, L, dtype=np.uint8), (N, 1))
    else:
        msa = np.repeat(rng.integers(0, 21, (N, 1), dtype=np.uint8), L, axis=1)
    w = oracle_mod.oracle_weights(msa, 0.8)
    for xkind in ("bias", "rand"):
        if xkind == "bias":
            from ccmpred_b200.host import init_bias
            x = init_bias(msa)
        else:
            x = synth.random_x(L, 18)
        f, g = run(path, msa, w, x, 0.01, 0.2 * (L - 1))
        assert np.all(np.isfinite(g))
        f64, g64 = oracle_mod.oracle_evaluate(msa, w, 0.01, 0.2 * (L - 1), x)
        e = errors(f, g, f64, g64, L)
        assert within(e, TOL[path]), (xkind, e)


@pytest.mark.parametrize("path", ["tc_bf16x2", "tc_i8x3", "tc_i8sp", "simt_f32"])
def test_inadmissible_x(gpu, oracle_mod, path):
    """Non-zero padding states and self blocks: g follows the CPU reference
    (2*lambda2*x there, g1 padding zero)."""
    msa = synth.generate(synth.MSAConfig("t", 11, 40, seed=3))
    L = 11
    x = np.random.default_rng(1).normal(0, 0.03, oracle_mod.nvar_padded(L)).astype(np.float32)
    w = np.ones(40, np.float32)
    f, g = run(path, msa, w, x, 0.01, 2.0)
    f64, g64 = oracle_mod.oracle_evaluate(msa, w, 0.01, 2.0, x)
    e = errors(f, g, f64, g64, L)
    assert within(e, TOL[path]), e


def test_weights_bit_exact(gpu, oracle_mod):
    d = np.load(os.path.join(GOLDEN, "weights_L40_N300_dup.npz"))
    for t in d["thresholds"]:
        w = calculate_weights(d["msa"], float(t))
        assert np.array_equal(w.view(np.uint32), d[f"w_{int(round(float(t) * 100))}"].view(np.uint32))
    msa = synth.generate(synth.MSAConfig("t", 203, 1500, gap_frac=0.2, dup_frac=0.3, seed=8))
    for t in (0.8, 0.62):
        a = calculate_weights(msa, t)
        b = oracle_mod.oracle_weights(msa, t)
        assert np.array_equal(a.view(np.uint32), b.view(np.uint32))


def test_reference_triple(gpu, oracle_mod):
    """init_cuda / evaluate_cuda / destroy_cuda with the reference userdata layout."""
    import torch
    msa = synth.generate(synth.MSAConfig("t", 20, 150, n_pairs=3, dup_frac=0.3, seed=31))
    N, L = msa.shape
    ud = _lib.CcmUserdata()
    ud.msa = msa.ctypes.data_as(ctypes.POINTER(ctypes.c_ubyte))
    wbuf = np.zeros(N, dtype=np.float32)
    ud.weights = wbuf.ctypes.data_as(ctypes.POINTER(ctypes.c_float))
    ud.ncol, ud.nrow, ud.nsingle = L, N, 20 * L
    ud.nvar = 20 * L + 441 * L * L
    ud.lambda_single, ud.lambda_pair, ud.reweighting_threshold = 0.01, 0.2 * (L - 1), 0.8
    assert lib().init_cuda(ctypes.byref(ud)) == 0
    assert np.array_equal(wbuf.view(np.uint32), oracle_mod.oracle_weights(msa, 0.8).view(np.uint32))
    x = synth.random_x(L, 5)
    xd = torch.from_numpy(x).cuda()
    gd = torch.empty_like(xd)
    f = lib().evaluate_cuda(ctypes.byref(ud), xd.data_ptr(), gd.data_ptr(), x.size)
    f64, g64 = oracle_mod.oracle_evaluate(msa, wbuf, 0.01, 0.2 * (L - 1), x)
    e = errors(f, gd.cpu().numpy(), f64, g64, L)
    assert within(e, TOL["tc_bf16x2"]), e
    # host-pointer variant on a second instance
    ud2 = _lib.CcmUserdata.from_buffer_copy(ud)
    ud2.extra = None
    assert lib().init_b200(ctypes.byref(ud2)) == 1
    gh = np.empty_like(x)
    f2 = lib().evaluate_b200(ctypes.byref(ud2), x.ctypes.data_as(ctypes.POINTER(ctypes.c_float)),
                             gh.ctypes.data_as(ctypes.POINTER(ctypes.c_float)), x.size)
    assert f2 == f and np.array_equal(gh, gd.cpu().numpy())
    assert lib().destroy_b200(ctypes.byref(ud2)) == 0
    assert lib().destroy_cuda(ctypes.byref(ud)) == 0


@pytest.mark.parametrize("path", ["tc_bf16x2", "tc_i8x3", "tc_i8sp"])
def test_errors_and_determinism(gpu, path):
    import torch
    msa = synth.generate(synth.MSAConfig("t", 30, 200, seed=4))
    ev = Evaluator(msa, path=path)
    x = torch.from_numpy(synth.random_x(30, 1)).cuda()
    g = torch.empty_like(x)
    rc = lib().ccm_evaluate(ev.handle, x.data_ptr(), g.data_ptr(), x.numel() - 1, None)
    assert rc == _lib.CCM_ERR_INVALID and b"nvar" in lib().ccm_last_error()
    f1 = ev.evaluate(x, g)
    g1 = g.clone()
    f2 = ev.evaluate(x, g)
    assert f1 == f2 and torch.equal(g, g1)   # bit-for-bit deterministic
    ev.close()


@pytest.mark.parametrize("path", ["tc_i8sp", "tc_i8x3"])
def test_long_alignment_against_f64_path(gpu, path):
    """L = 700, a long alignment (prep stages rows of ~15k slots in shared memory, the
    backward's slot space is ~59 pair-tile blocks, K = 14700 for the sparse forward),
    checked against the FP64 CUDA-core path, itself checked against the oracle above."""
    import torch
    msa = synth.generate(synth.MSAConfig("t", 700, 96, n_pairs=20, seed=21))
    N, L = msa.shape
    w = calculate_weights(msa, 0.8)
    x = synth.random_x(L, 22)
    xd = torch.from_numpy(x).cuda()
    ref = Evaluator(msa, weights=w, path="simt_f64")
    g64 = torch.empty_like(xd, dtype=torch.float64)
    f64 = ref.evaluate(xd.double(), g64)
    ref.close()
    ev = Evaluator(msa, weights=w, path=path)
    g = torch.full_like(xd, float("nan"))
    f = ev.evaluate(xd, g)
    ev.close()
    e = errors(f, g.cpu().numpy(), f64, g64.cpu().numpy(), L)
    assert within(e, TOL[path]), e


@pytest.mark.parametrize("path", ["tc_i8sp", "simt_f32"])
def test_host_pointer_evaluation_and_padding(gpu, path):
    """ccm_evaluate_host equals the device-pointer evaluation bit for bit in every
    case of its padding rule: zero padding states (they and g's stay off PCIe, g's
    written as zeros on the host: fewer bytes copied), nonzero padding (an
    inadmissible x: copied both ways), zero again after that (the device copy's
    padding cleared), and -0.0 in the padding (a nonzero bit pattern: copied)."""
    import torch
    L, N = 37, 300
    msa = synth.generate(synth.MSAConfig("hp", L, N, n_pairs=3, seed=41))
    nsp = 20 * L + 32 - (20 * L) % 32
    x0 = synth.random_x(L, 42)
    x1 = x0.copy()
    x1[nsp:].reshape(21, L, 32, L)[:, :, 21:, :] = 0.01 * np.random.default_rng(43).standard_normal(
        (21, L, 11, L)).astype(np.float32)
    x2 = x0.copy()
    x2[nsp + 5 * 32 * L + 21 * L + 3] = -0.0
    real = 4 * (nsp + 21 * L * 21 * L)
    full = 4 * x0.size
    with Evaluator(msa, path=path) as ev:
        for x, h2d_expected in ((x0, real), (x1, full), (x0, real), (x2, full)):
            xd = torch.from_numpy(x).cuda()
            gd = torch.empty_like(xd)
            f_dev = ev.evaluate(xd, gd)
            gh = np.full_like(x, np.nan)
            f_host = ev.evaluate(np.ascontiguousarray(x), gh)
            assert f_host == f_dev
            assert np.array_equal(gh.view(np.uint32), gd.cpu().numpy().view(np.uint32))
            h2d, d2h = ctypes.c_longlong(), ctypes.c_longlong()
            assert lib().ccm_host_copy_bytes(ev.handle, ctypes.byref(h2d), ctypes.byref(d2h)) == 0
            assert h2d.value == h2d_expected and d2h.value == h2d_expected + 32
