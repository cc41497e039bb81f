"""The write set of the backward's output phase (CPU restatement of the index
arithmetic of i8_backward_kernel / tc_backward_kernel's epilogue): with the tied
gradient every coupling entry (b, k, a, j) with k != j receives exactly one
addition -- the symmetric tile value T[s1][s2] = G2[s1][s2] + G2[s2][s1] goes to
the entry whose row slot is the smaller one directly and to its mirror from the
same tile -- self blocks (k == j) none, and every single-field entry g1(b, k),
b < 20, exactly one store from the ones slot.  With the partial-derivative
gradient every entry, self blocks included, gets one addition.  One addition per
entry on top of prep's 2 lambda2 x is why the atomic adds give the same float in
any order."""
import numpy as np
import pytest

Q = 21


def slot_groups(cols, slots):
    return dict(cols=cols, slots=slots, used=Q * cols, ones=Q * cols)


def decode(s, G, L):
    """slot -> (state, column, valid): s = (l // cols) * slots + q * cols + l % cols."""
    t, r = s // G["slots"], s % G["slots"]
    q, l = r // G["cols"], t * G["cols"] + r % G["cols"]
    return q, l, (r < G["used"]) & (l < L)


def write_counts(L, G, sym):
    groups = (L + G["cols"] - 1) // G["cols"]
    S = (groups * G["slots"] + 255) // 256 * 256
    blocks = S // 256
    tiles = [(P, Qb) for Qb in range(blocks) for P in range(blocks) if not sym or P <= Qb]
    g2 = np.zeros((Q, L, Q, L), dtype=np.int64)       # (b, k, a, j)
    g1 = np.zeros((Q - 1, L), dtype=np.int64)
    for P, Qb in tiles:
        # all 256 row slots of the pair (CTA rank, warp quarter, lane) against the
        # 256 column slots (warp half, 8-column blocks): one (s1, s2) grid per tile
        s1 = P * 256 + np.arange(256)[:, None]
        s2 = Qb * 256 + np.arange(256)[None, :]
        b, k, v1 = decode(s1, G, L)
        a, j, v2 = decode(s2, G, L)
        s1b, s2b = np.broadcast_to(s1, (256, 256)), np.broadcast_to(s2, (256, 256))
        if sym:
            # mirrored writes: s1 < s2 -> entry (a, j, b, k); the ones column -> g1(b, k)
            m = (s1b < s2b) & v1 & v2 & (k != j)
            np.add.at(g2, (np.broadcast_to(a, m.shape)[m], np.broadcast_to(j, m.shape)[m],
                           np.broadcast_to(b, m.shape)[m], np.broadcast_to(k, m.shape)[m]), 1)
            o = (s1b < s2b) & ~(v1 & v2) & (s2b == G["ones"]) & v1 & (b < Q - 1)
            np.add.at(g1, (np.broadcast_to(b, o.shape)[o], np.broadcast_to(k, o.shape)[o]), 1)
        # direct writes: s1 <= s2 (tied) or every pair (partial) -> entry (b, k, a, j);
        # the ones row -> g1(a, j)
        keep = (s1b <= s2b) if sym else np.ones((256, 256), bool)
        d = keep & v1 & v2 & ((k != j) if sym else True)
        np.add.at(g2, (np.broadcast_to(b, d.shape)[d], np.broadcast_to(k, d.shape)[d],
                       np.broadcast_to(a, d.shape)[d], np.broadcast_to(j, d.shape)[d]), 1)
        o = keep & ~v1 & (s1b == G["ones"]) & v2 & (a < Q - 1)
        np.add.at(g1, (np.broadcast_to(a, o.shape)[o], np.broadcast_to(j, o.shape)[o]), 1)
    return g2, g1


@pytest.mark.parametrize("G", [slot_groups(9, 192), slot_groups(12, 256)],
                         ids=["groups192", "groups256"])
@pytest.mark.parametrize("L", [1, 2, 9, 10, 13, 25, 40])
def test_tied_gradient_gets_one_addition_per_entry(L, G):
    g2, g1 = write_counts(L, G, sym=True)
    self_block = np.eye(L, dtype=bool)[None, :, None, :]
    assert np.all(g2[np.broadcast_to(~self_block, g2.shape)] == 1)
    assert np.all(g2[np.broadcast_to(self_block, g2.shape)] == 0)
    assert np.all(g1 == 1)


@pytest.mark.parametrize("G", [slot_groups(9, 192), slot_groups(12, 256)],
                         ids=["groups192", "groups256"])
@pytest.mark.parametrize("L", [1, 9, 13, 25])
def test_partial_gradient_gets_one_addition_per_entry(L, G):
    g2, g1 = write_counts(L, G, sym=False)
    assert np.all(g2 == 1)
    assert np.all(g1 == 1)
