"""Numpy restatement of the sparse integer path's operand layouts (tc_i8sp), shared
by the CPU layout test and the GPU stage test.

K order of the forward: k' = l * 21 + q (alignment column major), KP = 21 L padded to
256.  Slot groups of the backward and of the forward's N: 9 columns per 192 slots,
s(q, l) = (l // 9) * 192 + q * 9 + l % 9, ones slot 189.  The forward's operands are
stored as tiled shared-memory images (swizzle included); the index maps below give
the byte of the stored array for each logical (row, column)."""
import numpy as np

Q = 21


def slot192(q, l):
    return (l // 9) * 192 + q * 9 + (l % 9)


def sp_shapes(L, N):
    T = (L + 8) // 9
    SW = 192 * T
    S = (SW + 255) // 256 * 256
    KP = (Q * L + 255) // 256 * 256
    Npad = (N + 255) // 256 * 256
    return T, SW, S, KP, Npad


def sp_a_index(Npad, KP):
    """Compressed one-hot: 128 rows x 64 bytes per 128 logical K, 64-byte swizzle."""
    n = np.arange(Npad)[:, None]
    col = np.arange(KP // 2)[None, :]
    KB = KP // 128
    r = n & 127
    return ((((n >> 7) * KB + (col >> 6)) * 128 + r) * 64
            + ((((col >> 4) & 3) ^ ((r >> 1) & 3)) << 4) + (col & 15))


def sp_e_index(Npad, KP):
    """2:4 metadata: 128 rows x 16 bytes per 128 logical K, no swizzle."""
    n = np.arange(Npad)[:, None]
    b = np.arange(KP // 8)[None, :]
    KB = KP // 128
    return (((n >> 7) * KB + (b >> 4)) * 128 + (n & 127)) * 16 + (b & 15)


def sp_b_index(KP, SW):
    """Digits of W: per forward tile and CTA half, 128 K rows x 96 slots as three
    32-slot atoms, 32-byte swizzle."""
    kr = np.arange(KP)[:, None]
    s = np.arange(SW)[None, :]
    KB = KP // 128
    t, c = s // 192, s % 192
    h, i, xx, r = c // 96, (c % 96) >> 5, c & 31, kr & 127
    return (((((t * 2 + h) * KB + (kr >> 7)) * 3 + i) * 4096 + r * 32
             + ((((xx >> 4) ^ (r >> 2)) & 1) << 4) + (xx & 15)))


def sp_bwd_index(Npad, S):
    """The backward's operands (one-hot x1 / x128, digits of R), Npad x S: 32-row x
    128-slot tiles (kb = n // 32, sb = s // 128) of 4 KB in the order sb * KB + kb,
    KB = Npad // 32; rows of 128 slots, 16-byte chunk c of row r at chunk c ^ (r & 7)."""
    n = np.arange(Npad)[:, None]
    s = np.arange(S)[None, :]
    KB = Npad // 32
    return (((s >> 7) * KB + (n >> 5)) * 4096 + (n & 31) * 128
            + (((((s & 127) >> 4) ^ (n & 7)) & 7) << 4) + (s & 15))


def onehot_natural(msa, KP, Npad):
    """O[n][l * 21 + q] = 1 where column l of row n holds state q."""
    N, L = msa.shape
    O = np.zeros((Npad, KP), dtype=np.int64)
    for l in range(L):
        O[np.arange(N), l * Q + msa[:, l].astype(np.int64)] = 1
    return O


def compress_2to4(O):
    """The builder's rule per group of four: the two kept positions i0 < i1 and
    their values (a single 1 keeps a zero partner: (p, 3) or (2, 3) for p = 3; an
    empty group keeps (0, 1)).  Returns (values [Npad, KP/2], i0, i1 [Npad, KP/4])."""
    Npad, KP = O.shape
    g = O.reshape(Npad, KP // 4, 4)
    assert g.sum(axis=2).max() <= 2
    i0 = np.zeros(g.shape[:2], dtype=np.int64)
    i1 = np.ones(g.shape[:2], dtype=np.int64)
    v = np.zeros(g.shape[:2] + (2,), dtype=np.int64)
    for n in range(Npad):
        for c in range(KP // 4):
            pos = np.flatnonzero(g[n, c])
            if len(pos) == 2:
                i0[n, c], i1[n, c] = pos
                v[n, c] = 1
            elif len(pos) == 1:
                p = pos[0]
                if p < 3:
                    i0[n, c], i1[n, c], v[n, c, 0] = p, 3, 1
                else:
                    i0[n, c], i1[n, c], v[n, c, 1] = 2, 3, 1
    return v.reshape(Npad, KP // 2), i0, i1


def decompress_2to4(vals, i0, i1):
    Npad, G = i0.shape
    out = np.zeros((Npad, G, 4), dtype=np.int64)
    rows = np.arange(Npad)[:, None]
    grp = np.arange(G)[None, :]
    out[rows, grp, i0] = vals[:, 0::2]
    out[rows, grp, i1] += vals[:, 1::2]
    return out.reshape(Npad, G * 4)
