"""ctypes binding of libccmpred_b200.so (the C ABI in include/ccmpred_b200.h).

The library is built in-tree by ``ccmpred_b200/csrc/Makefile`` (see
``ccmpred_b200.build``); loading it never falls back to anything else: a
missing library raises.
"""
from __future__ import annotations

import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libccmpred_b200.so")

CCM_OK = 0
CCM_ERR_INVALID = -1
CCM_ERR_CUDA = -2
CCM_ERR_NOMEM = -3
CCM_ERR_DEVICE = -4
CCM_ERR_UNSUPPORTED = -5

PATH_TC_BF16X2 = 0
PATH_TC_BF16X3 = 1
PATH_SIMT_F32 = 2
PATH_SIMT_F64 = 3
PATH_TC_I8X3 = 4
PATH_TC_I8SP = 5
PATHS = {"tc_bf16x2": PATH_TC_BF16X2, "tc_bf16x3": PATH_TC_BF16X3,
         "simt_f32": PATH_SIMT_F32, "simt_f64": PATH_SIMT_F64, "tc_i8x3": PATH_TC_I8X3,
         "tc_i8sp": PATH_TC_I8SP}


GRADIENT_TIED = 0
GRADIENT_PARTIAL = 1
GRADIENTS = {"tied": GRADIENT_TIED, "partial": GRADIENT_PARTIAL}


class CcmOptions(ctypes.Structure):
    _fields_ = [("lambda_single", ctypes.c_float), ("lambda_pair", ctypes.c_float),
                ("path", ctypes.c_int), ("device", ctypes.c_int), ("stream", ctypes.c_void_p),
                ("gradient", ctypes.c_int), ("max_sms", ctypes.c_int),
                ("mem_limit", ctypes.c_size_t)]


class CcmResult(ctypes.Structure):
    _fields_ = [("fx", ctypes.c_double), ("f_data", ctypes.c_double), ("reg", ctypes.c_double),
                ("status", ctypes.c_int), ("pad", ctypes.c_int)]


class CcmUserdata(ctypes.Structure):
    """Layout of the reference ``userdata`` (include/ccmpred.h:39-92)."""
    _fields_ = [("msa", ctypes.POINTER(ctypes.c_ubyte)), ("weights", ctypes.POINTER(ctypes.c_float)),
                ("ncol", ctypes.c_int), ("nrow", ctypes.c_int), ("nsingle", ctypes.c_int),
                ("nvar", ctypes.c_int), ("extra", ctypes.c_void_p),
                ("lambda_single", ctypes.c_float), ("lambda_pair", ctypes.c_float),
                ("reweighting_threshold", ctypes.c_float), ("meta_steps", ctypes.c_void_p)]


class CcmCgParams(ctypes.Structure):
    _fields_ = [("max_iterations", ctypes.c_int), ("k", ctypes.c_int),
                ("max_linesearch", ctypes.c_int), ("pad", ctypes.c_int),
                ("epsilon", ctypes.c_double), ("alpha_mul", ctypes.c_double),
                ("ftol", ctypes.c_double), ("wolfe", ctypes.c_double),
                ("min_gnorm", ctypes.c_double)]


class CcmCgResult(ctypes.Structure):
    _fields_ = [("status", ctypes.c_int), ("iterations", ctypes.c_int),
                ("evaluations", ctypes.c_int), ("pad", ctypes.c_int),
                ("fx", ctypes.c_double), ("gnorm", ctypes.c_double)]


CG_SUCCESS = 0
CG_ALREADY_MINIMIZED = 1
CG_STOPPED = 2
CG_ERR_MAXITER = -1023
CG_ERR_LINESEARCH = -1022
CG_ERR_NONFINITE = -1021

class CcmMsaDesc(ctypes.Structure):
    _fields_ = [("msa", ctypes.c_void_p), ("ncol", ctypes.c_int), ("nrow", ctypes.c_int),
                ("path", ctypes.c_int), ("pad", ctypes.c_int)]


class CcmBatchParams(ctypes.Structure):
    _fields_ = [("reweighting_threshold", ctypes.c_float), ("lambda_single", ctypes.c_float),
                ("lambda_pair_factor", ctypes.c_float), ("path", ctypes.c_int),
                ("workers", ctypes.c_int), ("device", ctypes.c_int), ("use_apc", ctypes.c_int),
                ("sms_per_worker", ctypes.c_int), ("waves", ctypes.c_int),
                ("wave_max", ctypes.c_int), ("wave_bytes", ctypes.c_size_t),
                ("cg", CcmCgParams)]


class CcmBatchResult(ctypes.Structure):
    _fields_ = [("status", ctypes.c_int), ("iterations", ctypes.c_int),
                ("evaluations", ctypes.c_int), ("pad", ctypes.c_int),
                ("fx", ctypes.c_double), ("seconds", ctypes.c_double)]


class ConjugradParams(ctypes.Structure):
    """conjugrad_parameter_t of include/conjugrad.h (float build)."""
    _fields_ = [("max_linesearch", ctypes.c_int), ("max_iterations", ctypes.c_int),
                ("k", ctypes.c_int), ("epsilon", ctypes.c_float), ("ftol", ctypes.c_float),
                ("wolfe", ctypes.c_float), ("alpha_mul", ctypes.c_float),
                ("min_gnorm", ctypes.c_float)]


CONJUGRAD_SUCCESS = 0
CONJUGRAD_ALREADY_MINIMIZED = 1
CONJUGRADERR_UNKNOWN = -1024
CONJUGRADERR_MAXIMUMITERATION = -1023
CONJUGRADERR_MAXIMUMLINESEARCH = -1022

# evaluate(instance, x, g, n) -> f  (conjugrad_evaluate_t)
EVALUATE = ctypes.CFUNCTYPE(ctypes.c_float, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                            ctypes.c_int)

# progress(instance, x, g, fx, xnorm, gnorm, step, n, k, ls) -> int
PROGRESS = ctypes.CFUNCTYPE(ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                            ctypes.c_float, ctypes.c_float, ctypes.c_float, ctypes.c_float,
                            ctypes.c_int, ctypes.c_int, ctypes.c_int)

# name -> (restype, argtypes); every symbol include/*.h declares
_vp = ctypes.c_void_p
_f32p = ctypes.POINTER(ctypes.c_float)
_f64p = ctypes.POINTER(ctypes.c_double)
_u8p = ctypes.POINTER(ctypes.c_ubyte)
SIGNATURES = {
    "ccm_nsingle_padded": (ctypes.c_longlong, [ctypes.c_int]),
    "ccm_nvar_padded": (ctypes.c_longlong, [ctypes.c_int]),
    "ccm_options_default": (None, [ctypes.POINTER(CcmOptions), ctypes.c_int]),
    "ccm_create": (ctypes.c_int, [ctypes.POINTER(_vp), _u8p, ctypes.c_int, ctypes.c_int, _f32p,
                                  ctypes.POINTER(CcmOptions)]),
    "ccm_destroy": (ctypes.c_int, [_vp]),
    "ccm_evaluate": (ctypes.c_int, [_vp, _vp, _vp, ctypes.c_longlong, _f64p]),
    "ccm_evaluate_async": (ctypes.c_int, [_vp, _vp, _vp, ctypes.c_longlong]),
    "ccm_evaluate_host": (ctypes.c_int, [_vp, _f32p, _f32p, ctypes.c_longlong, _f64p]),
    "ccm_evaluate_f64": (ctypes.c_int, [_vp, _vp, _vp, ctypes.c_longlong, _f64p]),
    "ccm_result_device": (_vp, [_vp]),
    "ccm_get_result": (ctypes.c_int, [_vp, ctypes.POINTER(CcmResult)]),
    "ccm_get_weights": (ctypes.c_int, [_vp, _f32p]),
    "ccm_stream": (_vp, [_vp]),
    "ccm_calculate_weights": (ctypes.c_int, [_u8p, ctypes.c_int, ctypes.c_int, ctypes.c_float,
                                             _f32p, ctypes.c_int]),
    "ccm_calculate_weights_noalloc": (ctypes.c_int, [_vp, ctypes.c_int, ctypes.c_int,
                                                     ctypes.c_float, _vp, _vp]),
    "ccm_last_error": (ctypes.c_char_p, []),
    "ccm_debug_copy": (ctypes.c_longlong, [_vp, ctypes.c_int, _vp, ctypes.c_longlong]),
    "ccm_profile_begin": (ctypes.c_int, [_vp, ctypes.c_int]),
    "ccm_profile_end": (ctypes.c_int, [_vp, _f64p, ctypes.c_int, ctypes.POINTER(ctypes.c_int),
                                       ctypes.POINTER(ctypes.c_int)]),
    "ccm_launch_count": (ctypes.c_longlong, [_vp]),
    "ccm_debug_set_wait_limit": (ctypes.c_int, [_vp, ctypes.c_longlong]),
    "ccm_debug_set_cg_skip_padding": (ctypes.c_int, [_vp, ctypes.c_int]),
    "ccm_host_copy_bytes": (ctypes.c_int, [_vp, ctypes.POINTER(ctypes.c_longlong),
                                           ctypes.POINTER(ctypes.c_longlong)]),
    "ccm_set_default_path": (None, [ctypes.c_int]),
    "ccm_cg_params_default": (None, [ctypes.POINTER(CcmCgParams)]),
    "ccm_conjugrad_gpu": (ctypes.c_int, [_vp, _vp, ctypes.c_longlong, ctypes.POINTER(CcmCgParams),
                                         PROGRESS, _vp, ctypes.POINTER(CcmCgResult)]),
    "ccm_conjugrad_host": (ctypes.c_int, [_vp, _f32p, ctypes.c_longlong, ctypes.POINTER(CcmCgParams),
                                          PROGRESS, _vp, ctypes.POINTER(CcmCgResult)]),
    "ccm_batch_params_default": (None, [ctypes.POINTER(CcmBatchParams)]),
    "ccm_solve_batch": (ctypes.c_int, [ctypes.c_int, ctypes.POINTER(CcmMsaDesc),
                                       ctypes.POINTER(CcmBatchParams),
                                       ctypes.POINTER(CcmBatchResult),
                                       ctypes.POINTER(ctypes.POINTER(ctypes.c_float))]),
    "ccm_device_count": (ctypes.c_int, []),
    "ccm_device_info": (ctypes.c_int, [ctypes.c_int, ctypes.c_char_p, ctypes.c_int,
                                       ctypes.POINTER(ctypes.c_size_t),
                                       ctypes.POINTER(ctypes.c_size_t)]),
    "ccm_init_bias": (None, [_u8p, ctypes.c_int, ctypes.c_int, _f32p]),
    "ccm_sum_submatrices": (ctypes.c_double, [_f32p, _f32p, ctypes.c_int]),
    "ccm_sum_submatrices_gpu": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int,
                                               ctypes.c_void_p]),
    "ccm_apc": (None, [_f32p, ctypes.c_int]),
    "ccm_normalize": (ctypes.c_int, [_f32p, ctypes.c_int]),
    "ccm_write_matrix": (ctypes.c_int, [ctypes.c_char_p, _f32p, ctypes.c_int, ctypes.c_int]),
    "ccm_write_raw": (ctypes.c_int, [ctypes.c_char_p, _f32p, ctypes.c_int]),
    "ccm_read_raw": (ctypes.c_int, [ctypes.c_char_p, _f32p, ctypes.c_int]),
    "ccm_read_msa": (_u8p, [ctypes.c_char_p, ctypes.POINTER(ctypes.c_int),
                            ctypes.POINTER(ctypes.c_int)]),
    "ccm_free": (None, [_vp]),
    "evaluate_cuda": (ctypes.c_float, [_vp, _vp, _vp, ctypes.c_int]),
    "init_cuda": (ctypes.c_int, [_vp]),
    "destroy_cuda": (ctypes.c_int, [_vp]),
    "evaluate_b200": (ctypes.c_float, [_vp, _f32p, _f32p, ctypes.c_int]),
    "init_b200": (ctypes.c_int, [_vp]),
    "destroy_b200": (ctypes.c_int, [_vp]),
    # include/conjugrad.h: the optimizer under libconjugrad's names
    "conjugrad_init": (ctypes.POINTER(ConjugradParams), []),
    "conjugrad_malloc": (_vp, [ctypes.c_int]),
    "conjugrad_free": (None, [_vp]),
    "conjugrad": (ctypes.c_int, [ctypes.c_int, _vp, _f32p, _vp, _vp, _vp,
                                 ctypes.POINTER(ConjugradParams)]),
    "conjugrad_gpu": (ctypes.c_int, [ctypes.c_int, _vp, _f32p, _vp, _vp, _vp,
                                     ctypes.POINTER(ConjugradParams)]),
}

_lib = None


class CcmError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"ccmpred_b200 error {code}: {msg}")
        self.code = code


def lib():
    """Load libccmpred_b200.so (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise FileNotFoundError(
                f"{LIB_PATH} not found: build it with `make -C ccmpred_b200/csrc` "
                "(or ccmpred_b200.build())")
        l = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(l, name)
            fn.restype = res
            fn.argtypes = args
        _lib = l
    return _lib


def check(rc: int) -> None:
    if rc != CCM_OK:
        raise CcmError(rc, lib().ccm_last_error().decode(errors="replace"))
