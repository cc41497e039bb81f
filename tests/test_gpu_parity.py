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

# relative error bounds vs FP64 (f, g1, g2).  The FP32 reference itself is
# within ~2e-6 of FP64 at these sizes (tests/test_oracle.py).
TOL = {
    "simt_f32": (1e-5, 1e-5, 1e-5),
    "tc_bf16x2": (1e-5, 1e-5, 1e-5),
    "tc_bf16x3": (1e-5, 1e-5, 1e-5),
}
PATHS = list(TOL)


def errors(f, g, f64, g64, L):
    nsp = nsingle_padded(L)
    ns = 20 * L

    def rel(a, b):
        return float(np.linalg.norm(a.astype(np.float64) - b) / max(np.linalg.norm(b), 1e-300))

    return (abs(f - f64) / abs(f64), rel(g[:ns], g64[:ns]), rel(g[nsp:], g64[nsp:]),
            float(np.abs(g.astype(np.float64) - g64).max() / np.abs(g64).max()))


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
    ef, e1, e2, _ = errors(f, g, f64, g64, msa.shape[1])
    tf, t1, t2 = TOL[path]
    assert ef < tf and e1 < t1 and e2 < t2, (ef, e1, e2)
    # against the reference's own FP32 output
    ef_r, e1_r, e2_r, _ = errors(f, g, float(d["f"]), d["g"].astype(np.float64), msa.shape[1])
    assert ef_r < tf + 2e-6 and e1_r < t1 + 2e-6 and e2_r < t2 + 2e-6


CASES = [
    ("L75_N1000_bias", synth.SMALL_75x1000, "bias"),
    ("L75_N1000_rand", synth.SMALL_75x1000, "rand"),
    ("L13_N64_rand", synth.MSAConfig("t", 13, 64, n_pairs=3, seed=13), "rand"),
    ("L1_N9_rand", synth.MSAConfig("t", 1, 9, seed=14), "rand"),
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
    ef, e1, e2, _ = errors(f, g, f64, g64, L)
    tf, t1, t2 = TOL[path]
    assert ef < tf and e1 < t1 and e2 < t2, (ef, e1, e2)


@pytest.mark.parametrize("path", ["tc_bf16x2", "simt_f32"])
def test_inadmissible_x(gpu, oracle_mod, path):
    """Non-zero padding states and self blocks: g follows the CPU reference
    (2*lambda2*x there, g1 padding zero)."""
    msa = synth.generate(synth.MSAConfig("t", 11, 40, seed=3))
    L = 11
    x = np.random.default_rng(1).normal(0, 0.03, oracle_mod.nvar_padded(L)).astype(np.float32)
    w = np.ones(40, np.float32)
    f, g = run(path, msa, w, x, 0.01, 2.0)
    f64, g64 = oracle_mod.oracle_evaluate(msa, w, 0.01, 2.0, x)
    ef, e1, e2, _ = errors(f, g, f64, g64, L)
    assert ef < 1e-5 and e1 < 1e-5 and e2 < 1e-5, (ef, e1, e2)


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
    ef, e1, e2, _ = errors(f, gd.cpu().numpy(), f64, g64, L)
    assert ef < 1e-5 and e1 < 1e-5 and e2 < 1e-5
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


def test_errors_and_determinism(gpu):
    import torch
    msa = synth.generate(synth.MSAConfig("t", 30, 200, seed=4))
    ev = Evaluator(msa)
    x = torch.from_numpy(synth.random_x(30, 1)).cuda()
    g = torch.empty_like(x)
    with pytest.raises(_lib.CcmError) as e:
        lib().ccm_evaluate(ev.handle, x.data_ptr(), g.data_ptr(), x.numel() - 1, None) and \
            _lib.check(lib().ccm_evaluate(ev.handle, x.data_ptr(), g.data_ptr(), x.numel() - 1, None))
        raise _lib.CcmError(-1, "unreachable")
    f1 = ev.evaluate(x, g)
    g1 = g.clone()
    f2 = ev.evaluate(x, g)
    assert f1 == f2 and torch.equal(g, g1)   # bit-for-bit deterministic
    ev.close()
