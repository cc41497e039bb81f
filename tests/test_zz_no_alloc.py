"""The allocation-free reweighting entry point, called through the C ABI.

ccm_calculate_weights_noalloc serves callers that cannot allocate device
memory (a memory pool that owns the GPU, or a pipeline that cannot take the
device-wide synchronisation of cudaFree): it keeps its scratch in a fixed
array inside the library.  Its weights must equal those of the allocating
entry point ccm_calculate_weights (which the other tests pin bit-exactly to
the reference's calculate_weights), on two calls in a row, so that the
scratch left over from the first call cannot leak into the second.

This file is collected last so that a run stopping at the first failure has
already run every other test; it also passes on its own in a fresh process.
"""
import ctypes

import numpy as np
import pytest

from ccmpred_b200 import _lib, calculate_weights, lib, synth

pytestmark = pytest.mark.gpu


def noalloc(d_msa, L, N, thr, d_w, stream):
    return lib().ccm_calculate_weights_noalloc(d_msa.data_ptr(), L, N, ctypes.c_float(thr),
                                               d_w.data_ptr(), stream)


def test_noalloc_weights_match_allocating_entry_point(gpu):
    import torch
    # two alignments of different sizes, so the second call runs over counts
    # that the first call left in the shared scratch
    cases = [
        (synth.generate(synth.MSAConfig("na1", 150, 3000, gap_frac=0.2, dup_frac=0.4, seed=41)), 0.8),
        (synth.generate(synth.MSAConfig("na2", 61, 1777, gap_frac=0.2, dup_frac=0.5, seed=42)), 0.62),
    ]
    stream = torch.cuda.current_stream()
    for msa, thr in cases:
        N, L = msa.shape
        expected = calculate_weights(msa, thr)
        d_msa = torch.from_numpy(msa).to(gpu)
        d_w = torch.full((N,), float("nan"), dtype=torch.float32, device=gpu)
        assert noalloc(d_msa, L, N, thr, d_w, stream.cuda_stream) == _lib.CCM_OK, \
            lib().ccm_last_error()
        stream.synchronize()
        got = d_w.cpu().numpy()
        assert np.array_equal(got.view(np.uint32), expected.view(np.uint32))


def test_noalloc_rejects_oversized_input(gpu):
    import torch
    d = torch.zeros(8, dtype=torch.uint8, device=gpu)
    w = torch.zeros(8, dtype=torch.float32, device=gpu)
    rc = lib().ccm_calculate_weights_noalloc(d.data_ptr(), 1, 262145, ctypes.c_float(0.8),
                                             w.data_ptr(), None)
    assert rc == _lib.CCM_ERR_INVALID
    assert b"exceeds the fixed scratch" in lib().ccm_last_error()


def test_noalloc_two_streams_ordered_by_an_event(gpu):
    """Calls on two streams share the scratch; an event that orders the second
    call after the first (the documented way to serialise them) gives both
    their exact weights."""
    import torch
    a = synth.generate(synth.MSAConfig("na3", 90, 2500, gap_frac=0.2, dup_frac=0.4, seed=43))
    b = synth.generate(synth.MSAConfig("na4", 47, 1200, gap_frac=0.1, dup_frac=0.6, seed=44))
    sa, sb = torch.cuda.Stream(), torch.cuda.Stream()
    outs = []
    for msa, thr, stream in ((a, 0.8, sa), (b, 0.7, sb)):
        N, L = msa.shape
        d_msa = torch.from_numpy(msa).to(gpu)
        d_w = torch.full((N,), float("nan"), dtype=torch.float32, device=gpu)
        torch.cuda.synchronize()
        outs.append((msa, thr, d_msa, d_w))
    done_a = torch.cuda.Event()
    msa, thr, d_msa, d_w = outs[0]
    assert noalloc(d_msa, msa.shape[1], msa.shape[0], thr, d_w, sa.cuda_stream) == _lib.CCM_OK
    done_a.record(sa)
    sb.wait_event(done_a)
    msa, thr, d_msa, d_w = outs[1]
    assert noalloc(d_msa, msa.shape[1], msa.shape[0], thr, d_w, sb.cuda_stream) == _lib.CCM_OK
    torch.cuda.synchronize()
    for msa, thr, _, d_w in outs:
        expected = calculate_weights(msa, thr)
        assert np.array_equal(d_w.cpu().numpy().view(np.uint32), expected.view(np.uint32))
