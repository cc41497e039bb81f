"""Exactness of the integer paths' digit arithmetic (CPU, exhaustive): the three
8-bit digits that i8_prep_kernel / the forward epilogue pack from a fixed-point
value q (21 fractional bits, clamped to [-2^21, 2^21)) -- d0 = q >> 14 as a signed
byte, d1 = (q >> 7) & 127, d2 = q & 127 -- give back q as d0 * 2^14 + (128 d1 + d2),
which is what the two s32 accumulators (hi: the d0 products; lo: the x128 one-hot
times d1 plus the one-hot times d2) hold per one-hot entry; and the accumulators
stay inside s32 at the sizes the kernels allow (the constants are read from
ccm_tc_i8.cu, so that a change of them is checked here)."""
import os
import re

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = open(os.path.join(ROOT, "ccmpred_b200", "csrc", "ccm_tc_i8.cu")).read()


def const(name):
    return int(re.search(rf"constexpr int {name} = (\d+);", SRC).group(1))


FRAC = const("kI8FracBits")
NARROW_MAX_L = const("kI8NarrowMaxL")
CHUNK_ROWS = const("kI8BwdChunkKB") * const("kI8BwdBK")


def digits(q):
    """The kernels' packing: low byte of each shifted value (byte_perm selector 0),
    d1 and d2 masked to 7 bits."""
    d0 = ((q >> 14) & 0xFF).astype(np.uint8).view(np.int8).astype(np.int64)
    d1 = (q >> 7) & 0x7F
    d2 = q & 0x7F
    return d0, d1, d2


def test_three_digits_reconstruct_every_clamped_value():
    q = np.arange(-(1 << FRAC), 1 << FRAC, dtype=np.int64)
    d0, d1, d2 = digits(q)
    assert d0.min() == -128 and d0.max() == 127
    assert d1.min() == 0 and d1.max() == 127 and d2.min() == 0 and d2.max() == 127
    hi, lo = d0, 128 * d1 + d2          # per one-hot entry: O1 * d0 and O128 * d1 + O1 * d2
    assert np.array_equal(hi * 16384 + lo, q)


def test_forward_merge_fits_32_bits_up_to_the_narrow_width():
    # a one-hot row holds L ones: |hi| <= 128 L, 0 <= lo <= 16383 L
    L = NARROW_MAX_L
    lo_max = 16383 * L
    assert -128 * L * 16384 >= -(1 << 31)
    assert 127 * L * 16384 + lo_max < (1 << 31)
    assert lo_max < (1 << 31)


def test_backward_chunk_fits_s32():
    # the symmetric backward adds two products per row to each accumulator entry
    # (O_P^T r_Q and r_P^T O_Q): per row |hi| <= 2 * 128 and 0 <= lo <= 2 * 16383
    n = CHUNK_ROWS
    assert 2 * 16383 * n < (1 << 31)
    assert 2 * 128 * n <= (1 << 31)
