"""ctypes front end of the oracle -- TEST INFRASTRUCTURE ONLY.

Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline leg import
this module.  It wraps two libraries built by ``oracle/Makefile``:

* ``oracle/libccmoracle.so`` -- the FP64 restatement in ``oracle/ccm_oracle.c``
  of ``src/evaluate_cpu.c:16-166`` and ``src/reweighting.c:9-58``;
* ``oracle/_ref/libccmref.so`` -- the reference's own C sources compiled in
  place (``evaluate_cpu``, ``evaluate_cpu_omp``, ``calculate_weights``,
  ``init_bias``, ``sum_submatrices``/``apc``/``normalize``, ``read_msa``,
  ``write_matrix``/``write_raw``/``read_raw``).

The reference functions use the reference's padded layout (``N_ALPHA_PAD`` =
32, ``include/ccmpred.h:5-17``), as does everything here.
"""
from __future__ import annotations

import ctypes
import os
import time
from typing import Optional

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "libccmoracle.so")
REF_SO = os.path.join(HERE, "_ref", "libccmref.so")
REF_CUDA_SO = os.path.join(HERE, "_ref", "libccmref_cuda.so")
# the reference's example alignment (example/1atzA.aln, L=75, N=3068), copied
# here by oracle/Makefile
REF_EXAMPLE_ALN = os.path.join(HERE, "_ref", "1atzA.aln")

Q = 21
QPAD = 32

_f32p = ctypes.POINTER(ctypes.c_float)
_f64p = ctypes.POINTER(ctypes.c_double)
_u8p = ctypes.POINTER(ctypes.c_ubyte)


def nsingle_padded(L: int) -> int:
    ns = L * (Q - 1)
    return ns + QPAD - ns % QPAD


def nvar_padded(L: int) -> int:
    return nsingle_padded(L) + L * L * Q * QPAD


def _ptr(a: np.ndarray, t):
    return a.ctypes.data_as(t)


_oracle = None
_ref = None


def build() -> None:
    """Build the oracle libraries (and the reference ones, when its checkout exists)."""
    import subprocess
    subprocess.run(["make", "-s", "-C", HERE, "all"], check=True)


def oracle_lib():
    global _oracle
    if _oracle is None:
        if not os.path.exists(ORACLE_SO):
            build()
        lib = ctypes.CDLL(ORACLE_SO)
        lib.oracle_evaluate_f64.restype = ctypes.c_double
        lib.oracle_evaluate_f64.argtypes = [_u8p, _f64p, ctypes.c_int, ctypes.c_int,
                                            ctypes.c_double, ctypes.c_double, _f64p, _f64p]
        lib.oracle_calculate_weights.restype = None
        lib.oracle_calculate_weights.argtypes = [_u8p, ctypes.c_int, ctypes.c_int,
                                                 ctypes.c_float, _f32p]
        lib.oracle_conjugrad_f64.restype = ctypes.c_int
        lib.oracle_conjugrad_f64.argtypes = [_u8p, _f64p, ctypes.c_int, ctypes.c_int,
                                             ctypes.c_double, ctypes.c_double, _f64p,
                                             ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                             ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                             ctypes.c_double, _f64p,
                                             ctypes.POINTER(ctypes.c_int),
                                             ctypes.POINTER(ctypes.c_int)]
        lib.oracle_nvar_padded.restype = ctypes.c_long
        lib.oracle_nvar_padded.argtypes = [ctypes.c_int]
        _oracle = lib
    return _oracle


def ref_available() -> bool:
    return os.path.exists(REF_SO)


def ref_lib():
    global _ref
    if _ref is None:
        if not os.path.exists(REF_SO):
            raise FileNotFoundError(
                f"{REF_SO} is missing: build it with `make -C oracle ref` where the "
                "reference checkout is present")
        lib = ctypes.CDLL(REF_SO)
        vp = ctypes.c_void_p
        lib.ref_userdata_new.restype = vp
        lib.ref_userdata_new.argtypes = [_u8p, ctypes.c_int, ctypes.c_int,
                                         ctypes.c_float, ctypes.c_float, ctypes.c_float]
        lib.ref_userdata_weights.restype = _f32p
        lib.ref_userdata_weights.argtypes = [vp]
        lib.ref_userdata_free.argtypes = [vp]
        for name in ("init_cpu", "destroy_cpu", "init_cpu_omp", "destroy_cpu_omp"):
            getattr(lib, name).restype = ctypes.c_int
            getattr(lib, name).argtypes = [vp]
        for name in ("evaluate_cpu", "evaluate_cpu_omp"):
            getattr(lib, name).restype = ctypes.c_float
            getattr(lib, name).argtypes = [vp, _f32p, _f32p, ctypes.c_int]
        lib.init_bias.restype = None
        lib.init_bias.argtypes = [_f32p, vp]
        lib.calculate_weights.restype = None
        lib.calculate_weights.argtypes = [_f32p, _u8p, ctypes.c_uint64, ctypes.c_uint64,
                                          ctypes.c_float]
        lib.sum_submatrices.argtypes = [_f32p, _f32p, ctypes.c_int]
        lib.apc.argtypes = [_f32p, ctypes.c_int]
        lib.normalize.argtypes = [_f32p, ctypes.c_int]
        lib.read_raw.argtypes = [ctypes.c_char_p, vp, _f32p]
        lib.ref_read_msa_path.restype = ctypes.POINTER(ctypes.c_ubyte)
        lib.ref_read_msa_path.argtypes = [ctypes.c_char_p, ctypes.POINTER(ctypes.c_int),
                                          ctypes.POINTER(ctypes.c_int)]
        lib.ref_free.argtypes = [vp]
        lib.ref_write_matrix_path.argtypes = [ctypes.c_char_p, _f32p, ctypes.c_int, ctypes.c_int]
        lib.ref_write_raw_path.argtypes = [ctypes.c_char_p, _f32p, ctypes.c_int]
        _ref = lib
    return _ref


# ----------------------------------------------------------------------------- oracle (FP64)

def oracle_evaluate(msa: np.ndarray, weights: np.ndarray, lambda_single: float,
                    lambda_pair: float, x: np.ndarray):
    """(f, g) in float64 at x (any float dtype, padded layout)."""
    msa = np.ascontiguousarray(msa, dtype=np.uint8)
    N, L = msa.shape
    w = np.ascontiguousarray(weights, dtype=np.float64)
    x64 = np.ascontiguousarray(x, dtype=np.float64)
    assert x64.size == nvar_padded(L)
    g = np.empty_like(x64)
    f = oracle_lib().oracle_evaluate_f64(_ptr(msa, _u8p), _ptr(w, _f64p), L, N,
                                         float(lambda_single), float(lambda_pair),
                                         _ptr(x64, _f64p), _ptr(g, _f64p))
    return float(f), g


def oracle_conjugrad(msa, weights, lambda_single, lambda_pair, x0, max_iter=250, k=5,
                     max_ls=5, alpha_mul=0.5, ftol=float(np.float32(1e-4)),
                     wolfe=float(np.float32(0.2)), eps=0.01):
    """FP64 host CG with the rules of the device CG: (x, f_hist, iterations, evals, status).
    The defaults of ftol and wolfe are the reference's float values (src/ccmpred.c:532-533),
    as the device CG holds them."""
    msa = np.ascontiguousarray(msa, dtype=np.uint8)
    N, L = msa.shape
    w = np.ascontiguousarray(weights, dtype=np.float64)
    x = np.ascontiguousarray(x0, dtype=np.float64).copy()
    fh = np.zeros(max_iter + 1)
    it, ev = ctypes.c_int(0), ctypes.c_int(0)
    st = oracle_lib().oracle_conjugrad_f64(_ptr(msa, _u8p), _ptr(w, _f64p), L, N,
                                           lambda_single, lambda_pair, _ptr(x, _f64p), max_iter,
                                           k, max_ls, alpha_mul, ftol, wolfe, eps,
                                           _ptr(fh, _f64p), ctypes.byref(it), ctypes.byref(ev))
    return x, fh[: it.value + 1], it.value, ev.value, st


def oracle_weights(msa: np.ndarray, threshold: float) -> np.ndarray:
    msa = np.ascontiguousarray(msa, dtype=np.uint8)
    N, L = msa.shape
    w = np.empty(N, dtype=np.float32)
    oracle_lib().oracle_calculate_weights(_ptr(msa, _u8p), L, N, ctypes.c_float(threshold),
                                          _ptr(w, _f32p))
    return w


# ----------------------------------------------------------------------------- reference (FP32)

class RefEvaluator:
    """The reference's evaluate_cpu / evaluate_cpu_omp behind init/evaluate/destroy."""

    def __init__(self, msa: np.ndarray, lambda_single: float, lambda_pair: float,
                 threshold: float, omp: bool = False):
        self.lib = ref_lib()
        self.msa = np.ascontiguousarray(msa, dtype=np.uint8)
        self.N, self.L = self.msa.shape
        self.omp = omp
        self.ud = self.lib.ref_userdata_new(_ptr(self.msa, _u8p), self.L, self.N,
                                            lambda_single, lambda_pair, threshold)
        (self.lib.init_cpu_omp if omp else self.lib.init_cpu)(self.ud)
        self.nvar = nvar_padded(self.L)

    @property
    def weights(self) -> np.ndarray:
        p = self.lib.ref_userdata_weights(self.ud)
        return np.ctypeslib.as_array(p, shape=(self.N,)).copy()

    def evaluate(self, x: np.ndarray):
        x = np.ascontiguousarray(x, dtype=np.float32)
        g = np.empty_like(x)
        fn = self.lib.evaluate_cpu_omp if self.omp else self.lib.evaluate_cpu
        f = fn(self.ud, _ptr(x, _f32p), _ptr(g, _f32p), self.nvar)
        return float(f), g

    def close(self):
        if self.ud:
            # destroy_cpu frees ud->extra; destroy_cpu_omp leaks it (src/evaluate_cpu_omp.c:214-221)
            (self.lib.destroy_cpu_omp if self.omp else self.lib.destroy_cpu)(self.ud)
            self.lib.ref_userdata_free(self.ud)
            self.ud = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def ref_calculate_weights(msa: np.ndarray, threshold: float) -> np.ndarray:
    msa = np.ascontiguousarray(msa, dtype=np.uint8)
    N, L = msa.shape
    w = np.empty(N, dtype=np.float32)
    ref_lib().calculate_weights(_ptr(w, _f32p), _ptr(msa, _u8p), L, N, ctypes.c_float(threshold))
    return w


def ref_init_bias(msa: np.ndarray) -> np.ndarray:
    lib = ref_lib()
    msa = np.ascontiguousarray(msa, dtype=np.uint8)
    N, L = msa.shape
    ud = lib.ref_userdata_new(_ptr(msa, _u8p), L, N, 0.01, 0.2 * (L - 1), 0.8)
    x = np.empty(nvar_padded(L), dtype=np.float32)
    lib.init_bias(_ptr(x, _f32p), ud)
    lib.ref_userdata_free(ud)
    return x


def ref_read_msa(path: str) -> np.ndarray:
    lib = ref_lib()
    nc, nr = ctypes.c_int(0), ctypes.c_int(0)
    p = lib.ref_read_msa_path(path.encode(), ctypes.byref(nc), ctypes.byref(nr))
    if not p:
        raise FileNotFoundError(path)
    a = np.ctypeslib.as_array(p, shape=(nr.value * nc.value,)).copy().reshape(nr.value, nc.value)
    lib.ref_free(ctypes.cast(p, ctypes.c_void_p))
    return a


def ref_contact_map(x: np.ndarray, L: int, apc: bool = True, normalize: bool = False) -> np.ndarray:
    lib = ref_lib()
    x = np.ascontiguousarray(x, dtype=np.float32).copy()
    out = np.empty(L * L, dtype=np.float32)
    lib.sum_submatrices(_ptr(x, _f32p), _ptr(out, _f32p), L)
    if apc:
        lib.apc(_ptr(out, _f32p), L)
    if normalize:
        lib.normalize(_ptr(out, _f32p), L)
    return out.reshape(L, L)


def ref_write_matrix(path: str, mat: np.ndarray) -> None:
    mat = np.ascontiguousarray(mat, dtype=np.float32)
    ref_lib().ref_write_matrix_path(path.encode(), _ptr(mat, _f32p), mat.shape[1], mat.shape[0])


def ref_write_raw(path: str, x: np.ndarray, L: int) -> None:
    x = np.ascontiguousarray(x, dtype=np.float32)
    ref_lib().ref_write_raw_path(path.encode(), _ptr(x, _f32p), L)


def ref_read_raw(path: str, L: int) -> np.ndarray:
    lib = ref_lib()
    dummy = np.zeros((1, L), dtype=np.uint8)
    ud = lib.ref_userdata_new(_ptr(dummy, _u8p), L, 1, 0.01, 0.2 * (L - 1), 0.8)
    x = np.zeros(nvar_padded(L), dtype=np.float32)
    lib.read_raw(path.encode(), ud, _ptr(x, _f32p))
    lib.ref_userdata_free(ud)
    return x


class RefCudaEvaluator:
    """The reference's CUDA backend (src/evaluate_cuda.c + src/evaluate_cuda_kernels.cu,
    built for sm_100a by oracle/Makefile) behind init_cuda/evaluate_cuda/destroy_cuda.
    x and g are device pointers.  The reference keeps its device state in process
    globals: one instance per process at a time."""

    def __init__(self, msa: np.ndarray, lambda_single: float, lambda_pair: float,
                 threshold: float):
        lib = ctypes.CDLL(REF_CUDA_SO)
        vp = ctypes.c_void_p
        lib.ref_userdata_new.restype = vp
        lib.ref_userdata_new.argtypes = [_u8p, ctypes.c_int, ctypes.c_int,
                                         ctypes.c_float, ctypes.c_float, ctypes.c_float]
        lib.ref_userdata_free.argtypes = [vp]
        lib.init_cuda.argtypes = [vp]
        lib.destroy_cuda.argtypes = [vp]
        lib.evaluate_cuda.restype = ctypes.c_float
        lib.evaluate_cuda.argtypes = [vp, vp, vp, ctypes.c_int]
        self.lib = lib
        self.msa = np.ascontiguousarray(msa, dtype=np.uint8)
        self.N, self.L = self.msa.shape
        self.ud = lib.ref_userdata_new(_ptr(self.msa, _u8p), self.L, self.N,
                                       lambda_single, lambda_pair, threshold)
        lib.init_cuda(self.ud)
        self.nvar = nvar_padded(self.L)

    def evaluate(self, d_x: int, d_g: int) -> float:
        return float(self.lib.evaluate_cuda(self.ud, d_x, d_g, self.nvar))

    def close(self):
        if self.ud:
            self.lib.destroy_cuda(self.ud)
            self.lib.ref_userdata_free(self.ud)
            self.ud = None


def time_ref_evaluate(msa: np.ndarray, x: np.ndarray, lambda_single: float, lambda_pair: float,
                      threshold: float, omp: bool, repeats: int = 1,
                      budget_s: Optional[float] = None):
    """Seconds per evaluate call of the reference CPU path (median), and the call count."""
    ev = RefEvaluator(msa, lambda_single, lambda_pair, threshold, omp=omp)
    times = []
    try:
        t_start = time.perf_counter()
        for _ in range(repeats):
            t0 = time.perf_counter()
            ev.evaluate(x)
            times.append(time.perf_counter() - t0)
            if budget_s is not None and time.perf_counter() - t_start > budget_s:
                break
    finally:
        ev.close()
    return float(np.median(times)), len(times)
