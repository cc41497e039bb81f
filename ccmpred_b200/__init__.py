"""ccmpred_b200 -- CCMpred's pseudo-likelihood hot path on NVIDIA B200 (sm_100a).

The product is ``libccmpred_b200.so`` (CUDA kernels + C ABI declared in
``include/ccmpred_b200.h``).  This package is the Python mirror of that ABI,
used by the tests, the benchmark and the ``torch.autograd.Function`` wrapper:

* :class:`Evaluator` -- one alignment on the GPU; ``evaluate(x, g)`` is the
  reference's evaluate callback (``src/evaluate_cpu.c:16``,
  ``src/evaluate_cuda.c:23``) for device (torch CUDA tensors) or host (numpy)
  buffers in the reference's padded layout;
* :func:`calculate_weights` -- bit-exact GPU sequence reweighting
  (``src/reweighting.c:9-58``).
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from typing import Optional

import numpy as np

from . import _lib
from ._lib import CcmError, PATHS, check, lib

HERE = os.path.dirname(os.path.abspath(__file__))

N_ALPHA = 21
N_ALPHA_PAD = 32


def build(verbose: bool = False) -> str:
    """Compile libccmpred_b200.so in-tree for sm_100a (nvcc; no GPU needed)."""
    cmd = ["make", "-C", os.path.join(HERE, "csrc"), "-j8"]
    subprocess.run(cmd, check=True, stdout=None if verbose else subprocess.DEVNULL)
    return _lib.LIB_PATH


def nsingle_padded(L: int) -> int:
    ns = L * (N_ALPHA - 1)
    return ns + N_ALPHA_PAD - ns % N_ALPHA_PAD


def nvar_padded(L: int) -> int:
    return nsingle_padded(L) + L * L * N_ALPHA * N_ALPHA_PAD


def calculate_weights(msa: np.ndarray, threshold: float = 0.8, device: int = 0) -> np.ndarray:
    """Sequence weights on the GPU, bit-exact with the serial reference."""
    msa = np.ascontiguousarray(msa, dtype=np.uint8)
    N, L = msa.shape
    w = np.empty(N, dtype=np.float32)
    check(lib().ccm_calculate_weights(msa.ctypes.data_as(ctypes.POINTER(ctypes.c_ubyte)), L, N,
                                      ctypes.c_float(threshold),
                                      w.ctypes.data_as(ctypes.POINTER(ctypes.c_float)), device))
    return w


def solve_batch(msas, workers: int = 8, path: str = "tc_i8sp", threshold: float = 0.8,
                max_iterations: int = 250, epsilon: float = 0.01, contact_maps: bool = True,
                device: int = 0, sms_per_worker: int = 0, waves: bool = False,
                wave_max: int = 64, wave_bytes: int = 0):
    """Solve many alignments to convergence concurrently (ccm_solve_batch).

    ``path="auto"`` takes each alignment's path from the table that
    ``ccmpred_b200.autotune`` measured on the GPU.
    By default ``workers`` host threads with a context and stream each run the
    alignments' device-side solves; ``waves=True``: one graph launch per wave of
    alignments (``wave_max`` alignments at most, ``wave_bytes`` of device memory,
    0 = 60 % of the free memory).
    Returns (results, maps): per-alignment CcmBatchResult and APC contact maps."""
    arrs = [np.ascontiguousarray(m, dtype=np.uint8) for m in msas]
    n = len(arrs)
    table = None
    if path == "auto":
        # the per-size choice of ccmpred_b200.autotune (tuning_b200.json)
        from . import autotune
        table = autotune.load()
        if table is None:
            raise FileNotFoundError("path='auto' needs the table of ccmpred_b200.autotune "
                                    f"({autotune.TABLE}); run `python -m ccmpred_b200.autotune`")
    descs = (_lib.CcmMsaDesc * max(n, 1))()
    for i, a in enumerate(arrs):
        descs[i].msa = a.ctypes.data
        descs[i].nrow, descs[i].ncol = a.shape
        descs[i].path = PATHS[autotune.choose(table, a.shape[1], a.shape[0])] if table else -1
    p = _lib.CcmBatchParams()
    lib().ccm_batch_params_default(ctypes.byref(p))
    p.workers, p.reweighting_threshold, p.device = workers, threshold, device
    p.path = PATHS["tc_i8sp" if path == "auto" else path]
    p.sms_per_worker = sms_per_worker
    p.waves, p.wave_max, p.wave_bytes = int(bool(waves)), wave_max, wave_bytes
    p.cg.max_iterations, p.cg.epsilon = max_iterations, epsilon
    res = (_lib.CcmBatchResult * max(n, 1))()
    maps = [np.empty((a.shape[1], a.shape[1]), dtype=np.float32) for a in arrs] if contact_maps else None
    mptr = None
    if maps is not None:
        mptr = (ctypes.POINTER(ctypes.c_float) * max(n, 1))()
        for i, m in enumerate(maps):
            mptr[i] = m.ctypes.data_as(ctypes.POINTER(ctypes.c_float))
    check(lib().ccm_solve_batch(n, descs, ctypes.byref(p), res, mptr))
    return [res[i] for i in range(n)], maps


class Evaluator:
    """A ccm_context: the alignment, its weights and the device scratch of one path.

    ``path`` is one of ``tc_i8sp`` (default: 8-bit fixed-point digits, exact integer
    accumulation, the forward on 2:4-sparse MMAs), ``tc_i8x3`` (the same sums with a
    dense forward), ``tc_bf16x2``, ``tc_bf16x3``, ``simt_f32``, ``simt_f64``;
    ``gradient`` is ``tied`` (the reference's g, default) or ``partial`` (true
    partial derivatives, as autograd needs them); ``max_sms`` > 0 confines the
    tensor-core kernels to that many SMs (for contexts that share one GPU);
    ``mem_limit`` > 0 caps the context's device memory (bytes), beyond which
    creation or the optimizer fails with CCM_ERR_NOMEM.
    """

    def __init__(self, msa: np.ndarray, weights: Optional[np.ndarray] = None,
                 lambda_single: float = 0.01, lambda_pair: Optional[float] = None,
                 path: str = "tc_i8sp", device: int = 0, stream: Optional[int] = None,
                 gradient: str = "tied", max_sms: int = 0, mem_limit: int = 0):
        self._ctx = ctypes.c_void_p(None)
        self.msa = np.ascontiguousarray(msa, dtype=np.uint8)
        self.N, self.L = self.msa.shape
        self.path = path
        self.nvar = nvar_padded(self.L)
        self.nsp = nsingle_padded(self.L)
        self.lambda_single = float(lambda_single)
        # default as the reference computes it, in float: 0.2f * (L - 1)
        # (src/ccmpred.c:224,502-503)
        self.lambda_pair = float(np.float32(0.2) * np.float32(self.L - 1)
                                 if lambda_pair is None else lambda_pair)
        opt = _lib.CcmOptions()
        lib().ccm_options_default(ctypes.byref(opt), self.L)
        opt.lambda_single = self.lambda_single
        opt.lambda_pair = self.lambda_pair
        opt.path = PATHS[path]
        opt.device = device
        opt.stream = stream
        opt.gradient = _lib.GRADIENTS[gradient]
        opt.max_sms = max_sms
        opt.mem_limit = mem_limit
        self.gradient = gradient
        wptr = None
        if weights is not None:
            self.weights = np.ascontiguousarray(weights, dtype=np.float32)
            wptr = self.weights.ctypes.data_as(ctypes.POINTER(ctypes.c_float))
        check(lib().ccm_create(ctypes.byref(self._ctx),
                               self.msa.ctypes.data_as(ctypes.POINTER(ctypes.c_ubyte)),
                               self.L, self.N, wptr, ctypes.byref(opt)))
        if weights is None:
            self.weights = np.ones(self.N, dtype=np.float32)

    @property
    def handle(self) -> ctypes.c_void_p:
        return self._ctx

    @property
    def stream(self) -> int:
        return lib().ccm_stream(self._ctx)

    def evaluate(self, x, g) -> float:
        """f at x, gradient written into g.  x, g: torch CUDA tensors (float32, or
        float64 for the simt_f64 path) or numpy float32 host arrays."""
        fx = ctypes.c_double(0.0)
        if isinstance(x, np.ndarray):
            assert x.dtype == np.float32 and g.dtype == np.float32
            assert x.flags.c_contiguous and g.flags.c_contiguous
            check(lib().ccm_evaluate_host(self._ctx, x.ctypes.data_as(ctypes.POINTER(ctypes.c_float)),
                                          g.ctypes.data_as(ctypes.POINTER(ctypes.c_float)),
                                          x.size, ctypes.byref(fx)))
            return fx.value
        assert x.is_cuda and g.is_cuda and x.is_contiguous() and g.is_contiguous()
        if self.path == "simt_f64":
            check(lib().ccm_evaluate_f64(self._ctx, x.data_ptr(), g.data_ptr(), x.numel(),
                                         ctypes.byref(fx)))
        else:
            check(lib().ccm_evaluate(self._ctx, x.data_ptr(), g.data_ptr(), x.numel(),
                                     ctypes.byref(fx)))
        return fx.value

    def minimize(self, x, max_iterations: int = 250, epsilon: float = 0.01, k: int = 5,
                 progress=None, **kw) -> "_lib.CcmCgResult":
        """Device conjugate gradient from x (a float32 CUDA tensor, updated in place).

        ``progress(k, ls, fx, xnorm, gnorm, step)`` is called after every
        iteration; returning True stops the run."""
        p = _lib.CcmCgParams()
        lib().ccm_cg_params_default(ctypes.byref(p))
        p.max_iterations, p.epsilon, p.k = max_iterations, epsilon, k
        for name, val in kw.items():
            setattr(p, name, val)
        res = _lib.CcmCgResult()
        cb = _lib.PROGRESS(0)
        if progress is not None:
            def _cb(inst, xp, gp, fx, xnorm, gnorm, step, n, kk, ls):
                return 1 if progress(kk, ls, fx, xnorm, gnorm, step) else 0
            cb = _lib.PROGRESS(_cb)
        check(lib().ccm_conjugrad_gpu(self._ctx, x.data_ptr(), x.numel(), ctypes.byref(p), cb,
                                      None, ctypes.byref(res)))
        return res

    def evaluate_async(self, x, g) -> None:
        check(lib().ccm_evaluate_async(self._ctx, x.data_ptr(), g.data_ptr(), x.numel()))

    def result(self) -> "_lib.CcmResult":
        r = _lib.CcmResult()
        check(lib().ccm_get_result(self._ctx, ctypes.byref(r)))
        return r

    def close(self) -> None:
        if self._ctx:
            lib().ccm_destroy(self._ctx)
            self._ctx = ctypes.c_void_p(None)

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()
