"""The C-ABI library loads without a GPU and exports every symbol that
include/ccmpred_b200.h and include/conjugrad.h declare; the ctypes layouts
match the headers."""
import ctypes
import os
import re

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADERS = [os.path.join(ROOT, "include", h) for h in ("ccmpred_b200.h", "conjugrad.h")]


def declared_functions():
    text = "\n".join(open(h).read() for h in HEADERS)
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    text = re.sub(r"^\s*typedef[^;]*;", "", text, flags=re.M | re.S)
    names = re.findall(r"^\s*(?:const\s+)?[A-Za-z_][A-Za-z0-9_ ]*?[\s\*]+([a-z_][a-z0-9_]*)\s*\(",
                       text, flags=re.M)
    return sorted(set(n for n in names if not n.startswith("sizeof")))


def test_header_declares_the_reference_triple():
    names = declared_functions()
    for n in ("evaluate_cuda", "init_cuda", "destroy_cuda", "ccm_create", "ccm_evaluate",
              "ccm_calculate_weights", "ccm_destroy", "conjugrad_init", "conjugrad",
              "conjugrad_gpu", "conjugrad_malloc", "conjugrad_free"):
        assert n in names


def test_library_exports_every_declared_symbol():
    from ccmpred_b200 import _lib
    lib = _lib.lib()
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert missing == []
    # and the Python signature table covers the header
    assert sorted(_lib.SIGNATURES) == declared_functions()


def test_sizes_without_gpu():
    from ccmpred_b200 import _lib, nvar_padded, nsingle_padded
    lib = _lib.lib()
    for L in (1, 7, 12, 75, 300, 1000):
        assert lib.ccm_nsingle_padded(L) == nsingle_padded(L)
        assert lib.ccm_nvar_padded(L) == nvar_padded(L)
    # src/ccmpred.c:388-390 -- a full extra 32 when 20L is a multiple of 32
    assert nsingle_padded(8) == 160 + 32


def test_struct_layouts():
    from ccmpred_b200 import _lib
    assert ctypes.sizeof(_lib.CcmResult) == 32
    assert ctypes.sizeof(_lib.CcmOptions) == 40
    assert _lib.CcmOptions.mem_limit.offset == 32
    # reference userdata: 2 pointers, 4 ints, pointer, 3 floats, pointer (x86-64)
    assert ctypes.sizeof(_lib.CcmUserdata) == 64
    assert _lib.CcmUserdata.extra.offset == 32
    assert _lib.CcmUserdata.meta_steps.offset == 56


def test_userdata_layout_matches_reference(ref_mod):
    from ccmpred_b200 import _lib
    lib = ref_mod.ref_lib()
    lib.ref_sizeof_userdata.restype = ctypes.c_int
    assert lib.ref_sizeof_userdata() == ctypes.sizeof(_lib.CcmUserdata)


def test_errors_are_reported_without_gpu():
    from ccmpred_b200 import _lib
    lib = _lib.lib()
    msa = np.zeros((4, 3), dtype=np.uint8)
    ctx = ctypes.c_void_p()
    rc = lib.ccm_create(ctypes.byref(ctx), msa.ctypes.data_as(ctypes.POINTER(ctypes.c_ubyte)),
                        0, 4, None, None)
    assert rc == _lib.CCM_ERR_INVALID
    assert b"invalid" in lib.ccm_last_error()
    bad = np.full((4, 3), 21, dtype=np.uint8)
    rc = lib.ccm_create(ctypes.byref(ctx), bad.ctypes.data_as(ctypes.POINTER(ctypes.c_ubyte)),
                        3, 4, None, None)
    assert rc == _lib.CCM_ERR_INVALID
    assert b"state" in lib.ccm_last_error()


def test_batch_descriptor_layout_and_autotune_choice():
    from ccmpred_b200 import _lib, autotune
    assert ctypes.sizeof(_lib.CcmMsaDesc) == 24 and _lib.CcmMsaDesc.path.offset == 16
    table = {"buckets_L": [60, 200], "buckets_N": [300, 3000],
             "rows": [{"L": 60, "N": 300, "path": "simt_f32"},
                      {"L": 60, "N": 3000, "path": "tc_bf16x2"},
                      {"L": 200, "N": 300, "path": "tc_i8x3"},
                      {"L": 200, "N": 3000, "path": "tc_i8sp"}]}
    assert autotune.choose(table, 50, 250) == "simt_f32"
    assert autotune.choose(table, 60, 301) == "tc_bf16x2"
    assert autotune.choose(table, 61, 100) == "tc_i8x3"
    assert autotune.choose(table, 900, 90000) == "tc_i8sp"   # beyond the table: largest bucket
