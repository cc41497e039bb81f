"""The drop-in boundary: the reference's own driver (src/ccmpred.c, compiled
unchanged with -DCUDA by oracle/Makefile) linked against libccmpred_b200.so in
place of libconjugrad and the reference CUDA backend, and the libconjugrad
entry points (include/conjugrad.h) called directly.

The reference's own test (test/test.sh:1-9) runs its binary on
example/1atzA.aln and checks that the .mat has one line per column; the GPU
test here does that through this library and also checks that the .mat is
byte-identical to the one this repository's CLI writes with the same settings.
"""
import ctypes
import os
import re
import subprocess

import numpy as np
import pytest

from ccmpred_b200 import _lib, lib, nvar_padded, synth

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF_DRIVER = os.path.join(ROOT, "oracle", "_ref", "ccmpred-ref-b200")
CLI = os.path.join(ROOT, "ccmpred_b200", "ccmpred")
LETTERS = "ARNDCQEGHILKMFPSTWYV-"


def write_aln(path, msa):
    with open(path, "w") as f:
        for row in msa:
            f.write("".join(LETTERS[v] for v in row) + "\n")


def progress_f(stdout):
    """f(x) of the progress lines (src/ccmpred.c:62) in iteration order."""
    rows = [l.split("\t") for l in stdout.splitlines() if re.match(r"^\d+\s*\t", l)]
    return [float(r[2]) for r in rows]


@pytest.fixture(scope="module")
def ref_driver():
    if not os.path.exists(REF_DRIVER):
        pytest.skip("the reference driver was not built (oracle/Makefile with REF=...)")
    return REF_DRIVER


def test_conjugrad_init_defaults():
    p = lib().conjugrad_init()
    c = p.contents
    assert (c.max_linesearch, c.max_iterations, c.k) == (5, 250, 5)
    assert c.epsilon == np.float32(0.01) and c.ftol == np.float32(1e-4)
    assert c.wolfe == np.float32(0.2) and c.alpha_mul == 0.5 and c.min_gnorm == 0.0
    libc = ctypes.CDLL(None)
    libc.free.argtypes = [ctypes.c_void_p]
    libc.free(ctypes.cast(p, ctypes.c_void_p))   # the reference frees it (src/ccmpred.c:765)
    v = lib().conjugrad_malloc(1000)
    assert v and v % 64 == 0
    lib().conjugrad_free(v)


def test_conjugrad_host_vectors_match_fp64_cg(oracle_mod):
    """conjugrad() with host x and a host callback (here the FP64 oracle, rounded
    to float) applies the same rules as the FP64 restatement of the device CG."""
    msa = synth.generate(synth.MSAConfig("cgh", 10, 80, n_pairs=2, seed=81))
    N, L = msa.shape
    w = oracle_mod.oracle_weights(msa, 0.8)
    lam1, lam2 = 0.01, 0.2 * (L - 1)
    n = nvar_padded(L)
    x0 = oracle_mod.ref_init_bias(msa) if oracle_mod.ref_available() else None
    if x0 is None:
        from ccmpred_b200.host import init_bias
        x0 = init_bias(msa)
    iters = 8

    def evaluate(inst, xp, gp, nn):
        x = np.ctypeslib.as_array(ctypes.cast(xp, ctypes.POINTER(ctypes.c_float)), shape=(nn,))
        g = np.ctypeslib.as_array(ctypes.cast(gp, ctypes.POINTER(ctypes.c_float)), shape=(nn,))
        f, g64 = oracle_mod.oracle_evaluate(msa, w, lam1, lam2, x.astype(np.float64))
        g[:] = g64.astype(np.float32)
        return f

    seen = []

    def progress(inst, xp, gp, fx, xn, gn, st, nn, k, ls):
        seen.append(fx)
        return 0

    ev = _lib.EVALUATE(evaluate)
    pr = _lib.PROGRESS(progress)
    p = lib().conjugrad_init()
    p.contents.max_iterations = iters
    p.contents.epsilon = 0.0
    x = x0.astype(np.float32).copy()
    fx = ctypes.c_float()
    rc = lib().conjugrad(n, x.ctypes.data, ctypes.byref(fx), ctypes.cast(ev, ctypes.c_void_p),
                         ctypes.cast(pr, ctypes.c_void_p), None, p)
    assert rc == _lib.CONJUGRADERR_MAXIMUMITERATION
    _, fh, it_h, _, st_h = oracle_mod.oracle_conjugrad(msa, w, lam1, lam2, x0.astype(np.float64),
                                                       max_iter=iters, eps=0.0)
    assert it_h == iters and len(seen) == iters
    # float vectors against FP64 vectors: the same decisions, f to ~1e-6
    assert np.allclose(seen, fh[1:], rtol=1e-5)
    assert abs(fx.value - fh[-1]) / abs(fh[-1]) < 1e-5


def test_reference_driver_cpu_path(ref_driver, oracle_mod, tmp_path):
    """The reference's driver with -d -1 (its CPU path, src/ccmpred.c:636-648):
    this library's conjugrad around the reference's own evaluate_cpu."""
    msa = synth.generate(synth.MSAConfig("drv", 20, 150, n_pairs=3, dup_frac=0.2, seed=82))
    aln, mat = tmp_path / "in.aln", tmp_path / "out.mat"
    write_aln(aln, msa)
    r = subprocess.run([ref_driver, "-d", "-1", "-n", "4", str(aln), str(mat)],
                       capture_output=True, text=True, timeout=600, cwd=tmp_path)
    assert r.returncode == 0, r.stdout[-3000:] + r.stderr[-3000:]
    assert "Output can be found in" in r.stdout
    assert len(mat.read_text().splitlines()) == 20
    # the trajectory is the FP64 restatement's, to the reference's float precision
    w = oracle_mod.ref_calculate_weights(msa, 0.8)
    lam2 = float(np.float32(0.2) * np.float32(19))
    _, fh, it_h, _, _ = oracle_mod.oracle_conjugrad(msa, w, 0.01, lam2,
                                                    oracle_mod.ref_init_bias(msa).astype(np.float64),
                                                    max_iter=4, eps=float(np.float32(0.01)))
    # (the reference's evaluate_cpu sums f sequentially in float, src/evaluate_cpu.c:100,
    # which puts its f about 1e-4 off the FP64 value)
    f = progress_f(r.stdout)
    assert len(f) == it_h
    assert np.allclose(f, fh[1:], rtol=5e-4), (f, fh)


@pytest.mark.gpu
def test_reference_driver_on_example_alignment(gpu, ref_driver, oracle_mod, tmp_path):
    """test/test.sh through this library: the reference's binary on 1atzA.aln
    writes a 75-line .mat; it equals byte for byte the .mat of this repository's
    CLI at the same settings (both run the device CG on the same context type)."""
    aln = oracle_mod.REF_EXAMPLE_ALN
    if not os.path.exists(aln):
        pytest.skip("reference example alignment not copied into oracle/_ref")
    ref_mat, cli_mat = tmp_path / "ref.mat", tmp_path / "cli.mat"
    r = subprocess.run([ref_driver, "-n", "50", aln, str(ref_mat)], capture_output=True,
                       text=True, timeout=900, cwd=tmp_path)
    assert r.returncode == 0, r.stdout[-3000:] + r.stderr[-3000:]
    assert "using device #0" in r.stdout
    assert len(ref_mat.read_text().splitlines()) == 75
    c = subprocess.run([CLI, "-n", "50", aln, str(cli_mat)], capture_output=True, text=True,
                       timeout=900, cwd=tmp_path)
    assert c.returncode == 0, c.stdout[-3000:] + c.stderr[-3000:]
    assert progress_f(r.stdout) == progress_f(c.stdout)
    assert ref_mat.read_bytes() == cli_mat.read_bytes()


@pytest.mark.gpu
def test_conjugrad_gpu_routes_and_callbacks(gpu, tmp_path):
    """conjugrad_gpu with this library's evaluate_cuda and an init_cuda instance
    runs the fused device CG of ccm_conjugrad_gpu (same result bit for bit as
    calling it on an equal context); with a foreign callback (a Python function
    that evaluates through the C ABI) the same rules run around one callback call
    per trial and reach the same f to the precision of the float f it returns."""
    import torch
    from ccmpred_b200 import Evaluator
    from ccmpred_b200.host import init_bias
    msa = synth.generate(synth.MSAConfig("cgg", 40, 600, n_pairs=4, dup_frac=0.2, seed=83))
    N, L = msa.shape
    n = nvar_padded(L)
    lam2 = float(np.float32(0.2) * np.float32(L - 1))
    ud = _lib.CcmUserdata()
    ud.msa = msa.ctypes.data_as(ctypes.POINTER(ctypes.c_ubyte))
    wbuf = np.zeros(N, dtype=np.float32)
    ud.weights = wbuf.ctypes.data_as(ctypes.POINTER(ctypes.c_float))
    ud.ncol, ud.nrow, ud.nsingle, ud.nvar = L, N, 20 * L, 20 * L + 441 * L * L
    ud.lambda_single, ud.lambda_pair, ud.reweighting_threshold = 0.01, lam2, 0.8
    assert lib().init_cuda(ctypes.byref(ud)) == 0
    p = lib().conjugrad_init()
    p.contents.max_iterations = 15
    x0 = init_bias(msa)
    xa = torch.from_numpy(x0.copy()).cuda()
    fa = ctypes.c_float()
    evaluate_cuda = ctypes.cast(lib().evaluate_cuda, ctypes.c_void_p)
    rc = lib().conjugrad_gpu(n, xa.data_ptr(), ctypes.byref(fa), evaluate_cuda, None,
                             ctypes.byref(ud), p)
    assert rc in (_lib.CONJUGRAD_SUCCESS, _lib.CONJUGRADERR_MAXIMUMITERATION)
    with Evaluator(msa, weights=wbuf, lambda_pair=lam2) as ev:
        xb = torch.from_numpy(x0.copy()).cuda()
        res = ev.minimize(xb, max_iterations=15, epsilon=float(np.float32(0.01)))
        assert torch.equal(xa, xb) and fa.value == np.float32(res.fx)
        # a foreign callback: evaluates through ccm_evaluate, returns float f
        calls = [0]

        def evaluate(inst, xp, gp, nn):
            calls[0] += 1
            fx = ctypes.c_double()
            _lib.check(lib().ccm_evaluate(ev.handle, xp, gp, nn, ctypes.byref(fx)))
            return fx.value

        cb = _lib.EVALUATE(evaluate)
        xc = torch.from_numpy(x0.copy()).cuda()
        fc = ctypes.c_float()
        rc2 = lib().conjugrad_gpu(n, xc.data_ptr(), ctypes.byref(fc), ctypes.cast(cb, ctypes.c_void_p),
                                  None, None, p)
    assert rc2 in (_lib.CONJUGRAD_SUCCESS, _lib.CONJUGRADERR_MAXIMUMITERATION)
    assert calls[0] >= 15
    assert abs(fc.value - fa.value) / abs(fa.value) < 1e-4
    assert lib().destroy_cuda(ctypes.byref(ud)) == 0
