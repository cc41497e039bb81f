"""Failure detection, in the forms that fault no GPU: errors made on the host
(invalid inputs, a memory cap, a bad device number) and one bounded device wait
made to run out on a valid case.  The reference exits on every such error
(CHECK_ERR, include/evaluate_cuda_kernels.h:9; die, src/util.c:11-14); this
library returns status codes, which these tests check, and its CLI keeps the
reference's exits."""
import ctypes
import os
import subprocess

import numpy as np
import pytest

from ccmpred_b200 import CcmError, Evaluator, _lib, lib, nvar_padded, synth

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CLI = os.path.join(ROOT, "ccmpred_b200", "ccmpred")
LETTERS = "ARNDCQEGHILKMFPSTWYV-"


def create(msa, weights=None, **opt):
    """ccm_create through the C ABI; returns (status, context handle)."""
    msa = np.ascontiguousarray(msa, dtype=np.uint8)
    N, L = msa.shape
    o = _lib.CcmOptions()
    lib().ccm_options_default(ctypes.byref(o), L)
    for k, v in opt.items():
        setattr(o, k, v)
    ctx = ctypes.c_void_p()
    wptr = None
    if weights is not None:
        weights = np.ascontiguousarray(weights, dtype=np.float32)
        wptr = weights.ctypes.data_as(ctypes.POINTER(ctypes.c_float))
    rc = lib().ccm_create(ctypes.byref(ctx), msa.ctypes.data_as(ctypes.POINTER(ctypes.c_ubyte)),
                          L, N, wptr, ctypes.byref(o))
    return rc, ctx


# ---------------------------------------------------------------- host side (CPU)
def test_state_above_20_is_rejected():
    msa = synth.generate(synth.MSAConfig("t", 9, 30, seed=1))
    msa[17, 4] = 21
    rc, ctx = create(msa)
    assert rc == _lib.CCM_ERR_INVALID and not ctx.value
    assert b"MSA state 21" in lib().ccm_last_error()


@pytest.mark.parametrize("bad", [float("nan"), float("inf"), -float("inf")])
def test_non_finite_weight_is_rejected(bad):
    msa = synth.generate(synth.MSAConfig("t", 9, 30, seed=2))
    w = np.ones(30, np.float32)
    w[11] = bad
    rc, ctx = create(msa, weights=w)
    assert rc == _lib.CCM_ERR_INVALID and not ctx.value
    assert b"weight 11 is not finite" in lib().ccm_last_error()


def test_invalid_sizes_and_pointers_are_rejected():
    msa = np.zeros((4, 3), np.uint8)
    ctx = ctypes.c_void_p()
    assert lib().ccm_create(ctypes.byref(ctx), msa.ctypes.data_as(ctypes.POINTER(ctypes.c_ubyte)),
                            0, 4, None, None) == _lib.CCM_ERR_INVALID
    assert lib().ccm_create(ctypes.byref(ctx), None, 3, 4, None, None) == _lib.CCM_ERR_INVALID
    assert lib().ccm_debug_set_wait_limit(None, 0) == _lib.CCM_ERR_INVALID


def test_cli_bad_device_exits_like_the_reference(tmp_path):
    """-d outside the devices present: the reference prints an error and exits 1
    (src/ccmpred.c:410-413); without any device this program exits 1 too."""
    if not os.path.exists(CLI):
        pytest.skip("CLI not built")
    aln = tmp_path / "in.aln"
    msa = synth.generate(synth.MSAConfig("t", 12, 40, seed=3))
    aln.write_text("".join("".join(LETTERS[v] for v in row) + "\n" for row in msa))
    r = subprocess.run([CLI, "-d", "99", str(aln), str(tmp_path / "o.mat")], capture_output=True,
                       text=True, timeout=300)
    assert r.returncode == 1, r.stdout + r.stderr
    assert ("99 is not a valid device number" in r.stdout
            or "No CUDA devices available" in r.stderr)
    assert not (tmp_path / "o.mat").exists()


# ---------------------------------------------------------------- on the GPU
@pytest.mark.gpu
@pytest.mark.parametrize("path", ["tc_i8sp", "tc_i8x3", "tc_bf16x2", "simt_f32"])
@pytest.mark.parametrize("bad", [float("nan"), float("inf")])
def test_non_finite_x_gives_non_finite_f(gpu, path, bad):
    """A NaN or Inf in x is not an error of the evaluation: f comes back
    non-finite (as from the reference's evaluate_cpu), and the CG stops with
    CCM_CG_ERR_NONFINITE instead of iterating on it."""
    import torch
    msa = synth.generate(synth.MSAConfig("t", 20, 300, n_pairs=2, seed=4))
    x = synth.random_x(20, 5)
    L = 20
    x[nvar_padded(L) - 7 * L - 3] = bad     # a coupling
    with Evaluator(msa, path=path) as ev:
        xd = torch.from_numpy(x).cuda()
        gd = torch.empty_like(xd)
        f = ev.evaluate(xd, gd)
        assert not np.isfinite(f)
        x2 = synth.random_x(L, 6)
        x2[3 * L + 2] = bad                  # a single field
        xd2 = torch.from_numpy(x2).cuda()
        assert not np.isfinite(ev.evaluate(xd2, gd))
        res = ev.minimize(xd2, max_iterations=10)
        assert res.status == _lib.CG_ERR_NONFINITE and res.iterations == 0
        # the context is still usable
        x3 = torch.from_numpy(synth.random_x(L, 7)).cuda()
        assert np.isfinite(ev.evaluate(x3, gd)) and torch.isfinite(gd).all()


@pytest.mark.gpu
def test_memory_cap_gives_nomem(gpu):
    """ccm_options.mem_limit: the context counts the device memory it and its
    optimizer allocate; what does not fit fails with CCM_ERR_NOMEM and leaves
    nothing behind (the next context and evaluation work)."""
    import torch
    msa = synth.generate(synth.MSAConfig("t", 100, 1000, n_pairs=5, seed=8))
    L = 100
    # the tc_i8sp context needs about 31 MB at this size
    rc, ctx = create(msa, mem_limit=8 << 20)
    assert rc == _lib.CCM_ERR_NOMEM and not ctx.value, lib().ccm_last_error()
    # the context fits in 96 MB, the optimizer's four parameter-sized vectors
    # (4 x 27 MB) do not
    x = torch.from_numpy(synth.random_x(L, 9)).cuda()
    g = torch.empty_like(x)
    with Evaluator(msa, mem_limit=96 << 20) as ev:
        f_cap = ev.evaluate(x, g)
        g_cap = g.clone()
        with pytest.raises(CcmError) as err:
            ev.minimize(x.clone(), max_iterations=3)
        assert err.value.code == _lib.CCM_ERR_NOMEM
        assert ev.evaluate(x, g) == f_cap and torch.equal(g, g_cap)
    with Evaluator(msa) as ev:
        assert ev.evaluate(x, g) == f_cap and torch.equal(g, g_cap)
    with Evaluator(msa, mem_limit=512 << 20) as ev:
        res = ev.minimize(x.clone(), max_iterations=3)
        assert res.iterations == 3


@pytest.mark.gpu
@pytest.mark.parametrize("path", ["tc_i8sp", "tc_i8x3"])
def test_bounded_wait_runs_out(gpu, path):
    """The forward epilogue is made to wait 1000 clock cycles on a barrier that
    nothing arrives on: the wait gives up, the kernel records the timeout,
    drains its in-flight copies and MMAs, frees its tensor memory and returns;
    the evaluation reports CCM_ERR_DEVICE.  With the knob cleared the same
    context evaluates correctly again, bit for bit as a fresh one."""
    import torch
    msa = synth.generate(synth.MSAConfig("t", 60, 800, n_pairs=4, seed=10))
    x = torch.from_numpy(synth.random_x(60, 11)).cuda()
    g_ref = torch.empty_like(x)
    with Evaluator(msa, path=path) as ref:
        f_ref = ref.evaluate(x, g_ref)
    g = torch.empty_like(x)
    with Evaluator(msa, path=path) as ev:
        assert lib().ccm_debug_set_wait_limit(ev.handle, 1000) == _lib.CCM_OK
        fx = ctypes.c_double()
        rc = lib().ccm_evaluate(ev.handle, x.data_ptr(), g.data_ptr(), x.numel(), ctypes.byref(fx))
        assert rc == _lib.CCM_ERR_DEVICE, lib().ccm_last_error()
        assert b"timed out" in lib().ccm_last_error()
        assert lib().ccm_debug_set_wait_limit(ev.handle, 0) == _lib.CCM_OK
        assert ev.evaluate(x, g) == f_ref and torch.equal(g, g_ref)
    torch.cuda.synchronize()


def test_width_beyond_the_int_nvar_is_rejected():
    """L = 1788 makes nvar_padded exceed the reference ABI's int nvar (2^31 - 1):
    ccm_create refuses it before touching a device; L = 1787 is the widest."""
    from ccmpred_b200 import nvar_padded
    assert nvar_padded(1787) <= 0x7fffffff < nvar_padded(1788)
    msa = np.zeros((2, 1788), np.uint8)
    rc, ctx = create(msa)
    assert rc == _lib.CCM_ERR_INVALID and not ctx.value
    assert b"exceeds the int nvar" in lib().ccm_last_error()
