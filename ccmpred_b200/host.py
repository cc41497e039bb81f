"""Python mirror of the host-side C functions of libccmpred_b200.so
(``ccm_init_bias``, contact-map post-processing, file formats); each wraps the
C implementation, which restates the reference's host code bit-for-bit."""
from __future__ import annotations

import ctypes

import numpy as np

from ._lib import check, lib
from . import nvar_padded

_f32p = ctypes.POINTER(ctypes.c_float)
_u8p = ctypes.POINTER(ctypes.c_ubyte)


def init_bias(msa: np.ndarray) -> np.ndarray:
    """x0 of src/ccmpred.c:90-131 (single fields from column frequencies)."""
    msa = np.ascontiguousarray(msa, dtype=np.uint8)
    N, L = msa.shape
    x = np.empty(nvar_padded(L), dtype=np.float32)
    lib().ccm_init_bias(msa.ctypes.data_as(_u8p), L, N, x.ctypes.data_as(_f32p))
    return x


def contact_map(x: np.ndarray, L: int, apc: bool = True, normalize: bool = False):
    """(L x L map, xnorm): sum_submatrices, then optional APC and normalisation."""
    x = np.ascontiguousarray(x, dtype=np.float32)
    out = np.empty(L * L, dtype=np.float32)
    xnorm = lib().ccm_sum_submatrices(x.ctypes.data_as(_f32p), out.ctypes.data_as(_f32p), L)
    if apc:
        lib().ccm_apc(out.ctypes.data_as(_f32p), L)
    if normalize:
        check(lib().ccm_normalize(out.ctypes.data_as(_f32p), L))
    return out.reshape(L, L), xnorm


def write_matrix(path: str, mat: np.ndarray) -> None:
    mat = np.ascontiguousarray(mat, dtype=np.float32)
    check(lib().ccm_write_matrix(path.encode(), mat.ctypes.data_as(_f32p), mat.shape[1], mat.shape[0]))


def write_raw(path: str, x: np.ndarray, L: int) -> None:
    x = np.ascontiguousarray(x, dtype=np.float32)
    check(lib().ccm_write_raw(path.encode(), x.ctypes.data_as(_f32p), L))


def read_raw(path: str, L: int) -> np.ndarray:
    x = np.zeros(nvar_padded(L), dtype=np.float32)
    check(lib().ccm_read_raw(path.encode(), x.ctypes.data_as(_f32p), L))
    return x


def read_msa(path: str) -> np.ndarray:
    nc, nr = ctypes.c_int(0), ctypes.c_int(0)
    p = lib().ccm_read_msa(path.encode(), ctypes.byref(nc), ctypes.byref(nr))
    if not p:
        if nc.value == -1:
            raise ValueError(f"{path}: alignment seems to be in a3m or FASTA format; "
                             "PSICOV format expected")
        raise FileNotFoundError(path)
    a = np.ctypeslib.as_array(p, shape=(nr.value * nc.value,)).copy().reshape(nr.value, nc.value)
    lib().ccm_free(ctypes.cast(p, ctypes.c_void_p))
    return a
