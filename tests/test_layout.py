"""Structural properties of the sparse integer path's layouts (CPU): the 2:4 bound
that tcgen05.mma.sp relies on holds for every alignment in the K order l * 21 + q,
the builder's compression rule round-trips with valid metadata, the 192-slot groups
are a one-to-one slot map, and the tiled operand stores are bijections."""
import numpy as np
import pytest

from ccmpred_b200 import synth
from sparse_layout import (Q, compress_2to4, decompress_2to4, onehot_natural, slot192,
                           sp_a_index, sp_b_index, sp_bwd_index, sp_e_index, sp_shapes)


def adversarial_msa(L, N, seed):
    """Conserved columns, all-gap columns and runs of equal states next to random ones."""
    rng = np.random.default_rng(seed)
    msa = rng.integers(0, Q, size=(N, L), dtype=np.uint8)
    msa[:, ::3] = 20                      # all-gap columns
    msa[:, 1::5] = 7                      # conserved columns
    msa[: N // 2, 2::4] = msa[: N // 2, 2::4][:, :1]
    return msa


@pytest.mark.parametrize("L,N,seed", [(1, 9, 1), (5, 7, 2), (13, 64, 3), (40, 300, 4)])
def test_two_of_four(L, N, seed):
    for msa in (synth.generate(synth.MSAConfig("t", L, N, seed=seed)), adversarial_msa(L, N, seed)):
        _, _, _, KP, Npad = sp_shapes(L, N)
        O = onehot_natural(msa, KP, Npad)
        assert O.reshape(Npad, KP // 4, 4).sum(axis=2).max() <= 2
        vals, i0, i1 = compress_2to4(O)
        assert np.all(i0 < i1) and np.all(i1 <= 3)
        assert np.array_equal(decompress_2to4(vals, i0, i1), O)


@pytest.mark.parametrize("L", [1, 8, 9, 10, 300])
def test_groups192_slots(L):
    T, SW, S, KP, _ = sp_shapes(L, 1)
    s = np.array([[slot192(q, l) for l in range(L)] for q in range(Q)])
    assert len(np.unique(s)) == Q * L and s.max() < SW <= S and S % 256 == 0
    assert not np.any(s % 192 >= 189)   # slots 189..191 of a group: ones slot and padding
    assert KP % 256 == 0 and KP >= Q * L


@pytest.mark.parametrize("L,N", [(1, 9), (13, 50), (40, 300), (300, 5000)])
def test_tiled_stores_are_bijections(L, N):
    _, SW, S, KP, Npad = sp_shapes(L, N)
    for idx, size in ((sp_a_index(Npad, KP), Npad * KP // 2), (sp_e_index(Npad, KP), Npad * KP // 8),
                      (sp_b_index(KP, SW), KP * SW), (sp_bwd_index(Npad, S), Npad * S)):
        assert idx.size == size
        assert np.array_equal(np.sort(idx.ravel()), np.arange(size))


def test_backward_tile_rows_are_aligned_32_byte_pairs():
    """The forward epilogue writes 32 consecutive slots of one row of R as one
    32-byte store: in the backward's tiled storage those bytes form one aligned
    32-byte pair of 16-byte chunks (halves exchanged on odd rows mod 8)."""
    Npad, S = 512, 768
    idx = sp_bwd_index(Npad, S)
    for n in range(0, Npad, 7):
        for s0 in range(0, S, 32):
            b = idx[n, s0:s0 + 32]
            base = b.min()
            assert base % 32 == 0 and b.max() == base + 31
            lo_first = b[0] == base
            assert lo_first == ((n & 7) % 2 == 0)
