"""Stage-by-stage checks of the tensor-core path on small shapes: the one-hot
operand, the bf16 split of W in the slot layout, the forward GEMM + softmax
epilogue (through R) and the symmetric backward GEMM (through g), each
against a float64 numpy restatement of the same stage."""
import ctypes

import numpy as np
import pytest

from ccmpred_b200 import Evaluator, lib, synth
from sparse_layout import slot192, sp_a_index, sp_b_index, sp_bwd_index, sp_e_index

pytestmark = pytest.mark.gpu

Q, QP, G = 21, 32, 12


def slot(q, l):
    return (l // G) * 256 + q * G + (l % G)


def bf16_to_f32(u16):
    return (u16.astype(np.uint32) << 16).view(np.float32)


def fetch(ev, which, dtype=np.uint16):
    size = lib().ccm_debug_copy(ev.handle, which, None, 0)
    assert size > 0
    buf = np.empty(size // np.dtype(dtype).itemsize, dtype=dtype)
    assert lib().ccm_debug_copy(ev.handle, which, buf.ctypes.data, size) == 0
    return buf


def expected_internals(msa, w, x, L, lam2):
    N = msa.shape[0]
    T = (L + G - 1) // G
    S = T * 256
    Npad = (N + 255) // 256 * 256  # rows padded to the forward's 256-row pair tiles
    nsp = 20 * L + 32 - (20 * L) % 32
    V = x[:20 * L].reshape(20, L).astype(np.float64)
    W = x[nsp:].reshape(Q, L, QP, L)[:, :, :Q, :].astype(np.float64)      # [b,k,a,j]
    O = np.zeros((Npad, S))
    for n in range(N):
        for l in range(L):
            O[n, slot(int(msa[n, l]), l)] = 1.0
        O[n, 252] = 1.0
    Wp = np.zeros((S, S))
    sl = np.array([[slot(q, l) for l in range(L)] for q in range(Q)])   # [q,l]
    Wp[np.ix_(sl.reshape(-1), sl.reshape(-1))] = W.reshape(Q * L, Q * L)
    return O, Wp, V, sl, S, Npad


@pytest.mark.parametrize("path", ["tc_bf16x2", "tc_bf16x3"])
@pytest.mark.parametrize("L,N,seed", [(13, 50, 1), (24, 130, 2), (5, 7, 3)])
def test_tc_stages(gpu, path, L, N, seed):
    import torch
    msa = synth.generate(synth.MSAConfig("t", L, N, n_pairs=2, seed=seed))
    w = np.random.default_rng(seed).uniform(0.2, 1.0, N).astype(np.float32)
    x = synth.random_x(L, seed + 10, w_sd=0.05)
    lam2 = 0.2 * (L - 1)
    ev = Evaluator(msa, weights=w, lambda_pair=lam2, path=path)
    xd = torch.from_numpy(x).cuda()
    gd = torch.empty_like(xd)
    ev.evaluate(xd, gd)
    O, Wp, V, sl, S, Npad = expected_internals(msa, w, x, L, lam2)
    nsplit = 3 if path == "tc_bf16x3" else 2

    # one-hot operand, exact
    O_gpu = bf16_to_f32(fetch(ev, 0)).reshape(Npad, S)
    assert np.array_equal(O_gpu, O.astype(np.float32))

    # split terms of W: their sum reproduces W to the split's precision
    terms = [bf16_to_f32(fetch(ev, 1 + i)).reshape(S, S).astype(np.float64) for i in range(nsplit)]
    Wsum = sum(terms)
    tol = 2.0 ** (-16 if nsplit == 2 else -24)
    assert np.all(np.abs(Wsum - Wp) <= tol * np.abs(Wp) + 1e-30)

    # forward: logits from the split terms, softmax per (row, column), R
    logits = O[:N] @ Wsum                                   # [n, slot_out]
    R_exp = np.zeros((Npad, S))
    for l in range(L):
        cols = sl[:, l]
        z = logits[:, cols].copy()
        z[:, :20] += V[:, l][None, :]
        z -= z.max(axis=1, keepdims=True)
        P = np.exp(z) / np.exp(z).sum(axis=1, keepdims=True)
        onehot = (msa[:, l][:, None] == np.arange(Q)[None, :]).astype(np.float64)
        R_exp[:N, cols] = w[:, None] * (P - onehot)
    R_gpu = sum(bf16_to_f32(fetch(ev, 4 + i)).reshape(Npad, S).astype(np.float64)
                for i in range(nsplit))
    assert np.abs(R_gpu - R_exp).max() < 1e-5

    # backward: C = O^T R + R^T O from the GPU's own R, compared on g2
    C = O.T @ R_gpu + R_gpu.T @ O
    nsp = 20 * L + 32 - (20 * L) % 32
    g2 = gd.cpu().numpy()[nsp:].reshape(Q, L, QP, L).astype(np.float64)
    x2 = x[nsp:].reshape(Q, L, QP, L).astype(np.float64)
    G2 = C[np.ix_(sl.reshape(-1), sl.reshape(-1))].reshape(Q, L, Q, L)
    idx = np.arange(L)
    G2[:, idx, :, idx] = 0.0
    exp_g2 = 2 * np.float32(lam2) * x2.copy()
    exp_g2[:, :, :Q, :] += G2
    err = np.abs(g2 - exp_g2).max() / np.abs(exp_g2).max()
    assert err < 1e-5
    # single-field data gradient = column sums of R (ones slot of C)
    g1d = fetch(ev, 7, np.float32).reshape(20, L).astype(np.float64)
    g1_exp = R_gpu[:, sl[:20].reshape(-1)].sum(axis=0).reshape(20, L)
    assert np.abs(g1d - g1_exp).max() <= 1e-5 * max(1.0, np.abs(g1_exp).max())
    ev.close()


def digits_value(d0, d1, d2):
    """Integer Q of the three stored bytes: d0 signed, d1 and d2 in 0..127."""
    return d0.view(np.int8).astype(np.int64) * 16384 + d1.astype(np.int64) * 128 + d2.astype(np.int64)


@pytest.mark.parametrize("L,N,seed", [(13, 50, 1), (24, 130, 2), (5, 7, 3)])
def test_integer_path_stages(gpu, L, N, seed):
    """The integer path: column maxima of |W| exactly, the three digits of every
    W entry equal to clamp(rint(W * 2^(21 - e)), -2^21, 2^21 - 1) with e the
    column's exponent (bit-exact integers), the one-hot bytes, and the digits of R
    against an FP64 restatement of the forward at the quantised W (2^-21 abs)."""
    import torch
    msa = synth.generate(synth.MSAConfig("t", L, N, n_pairs=2, seed=seed))
    w = np.random.default_rng(seed).uniform(0.2, 1.0, N).astype(np.float32)
    x = synth.random_x(L, seed + 10, w_sd=0.05)
    lam2 = 0.2 * (L - 1)
    ev = Evaluator(msa, weights=w, lambda_pair=lam2, path="tc_i8x3")
    xd = torch.from_numpy(x).cuda()
    gd = torch.empty_like(xd)
    ev.evaluate(xd, gd)
    O, Wp, V, sl, S, Npad = expected_internals(msa, w, x, L, lam2)
    nsp = 20 * L + 32 - (20 * L) % 32
    W = x[nsp:].reshape(Q, L, QP, L)[:, :, :Q, :]                       # [b,k,a,j] float32

    # column maxima over rows (b,k) of |W(b,k,a,j)|, per column c = a*L + j
    cm = fetch(ev, 8, np.uint32).view(np.float32).reshape(Q, L)         # [a, j]
    assert np.array_equal(cm, np.abs(W).max(axis=(0, 1)))
    # exponent: smallest e with 2^e >= max (0 for an all-zero column)
    mant, ex = np.frexp(cm.astype(np.float64))                          # cm = mant * 2^ex, mant in [0.5,1)
    e = np.where(cm == 0, 0, np.where(mant == 0.5, ex - 1, ex))

    # one-hot bytes (x1 copy)
    O1 = fetch(ev, 0, np.uint8).reshape(Npad, S)
    assert np.array_equal(O1, O.astype(np.uint8))

    # digits of W in the slot layout, exact
    d = [fetch(ev, 1 + i, np.uint8).reshape(S, S) for i in range(3)]
    Qgpu = digits_value(*d)
    Qexp = np.zeros((S, S), dtype=np.int64)
    scale = np.ldexp(1.0, 21 - e)                                       # [a, j]
    Wq = np.clip(np.rint(W.astype(np.float64) * scale[None, None]), -2**21, 2**21 - 1)
    Qexp[np.ix_(sl.reshape(-1), sl.reshape(-1))] = Wq.astype(np.int64).reshape(Q * L, Q * L)
    assert np.array_equal(Qgpu, Qexp)

    # forward at the quantised W: logits, softmax, R = w (P - onehot); R digits at scale 1
    Wdeq = np.zeros((S, S))
    Wdeq[np.ix_(sl.reshape(-1), sl.reshape(-1))] = (Wq / scale[None, None]).reshape(Q * L, Q * L)
    logits = O[:N] @ Wdeq
    R_exp = np.zeros((Npad, S))
    for l in range(L):
        cols = sl[:, l]
        z = logits[:, cols].copy()
        z[:, :20] += V[:, l][None, :]
        z -= z.max(axis=1, keepdims=True)
        P = np.exp(z) / np.exp(z).sum(axis=1, keepdims=True)
        onehot = (msa[:, l][:, None] == np.arange(Q)[None, :]).astype(np.float64)
        R_exp[:N, cols] = w[:, None] * (P - onehot)
    r = [fetch(ev, 4 + i, np.uint8).reshape(Npad, S) for i in range(3)]
    R_gpu = digits_value(*r) / 2.0**21
    assert np.abs(R_gpu - R_exp).max() < 2.0**-21 + 2e-6
    ev.close()


@pytest.mark.parametrize("L,N,seed", [(13, 50, 1), (24, 130, 2), (5, 7, 3), (40, 300, 4)])
def test_sparse_integer_path_stages(gpu, L, N, seed):
    """The sparse integer path (tc_i8sp): the compressed one-hot operand of the
    forward decompresses to the one-hot in the K order l * 21 + q with valid 2:4
    metadata (two ascending positions per group of four); the digits of W sit in
    rows k * 21 + b and 192-slot-group columns (bit-exact); the one-hot of the
    backward and the digits of R use the 192-slot groups.  The forward's operands
    are read back through their tiled storage maps (each map a bijection)."""
    import torch
    msa = synth.generate(synth.MSAConfig("t", L, N, n_pairs=2, seed=seed))
    w = np.random.default_rng(seed).uniform(0.2, 1.0, N).astype(np.float32)
    x = synth.random_x(L, seed + 10, w_sd=0.05)
    lam2 = 0.2 * (L - 1)
    ev = Evaluator(msa, weights=w, lambda_pair=lam2, path="tc_i8sp")
    xd = torch.from_numpy(x).cuda()
    gd = torch.empty_like(xd)
    ev.evaluate(xd, gd)
    T = (L + 8) // 9
    SW = 192 * T
    S = (SW + 255) // 256 * 256
    KP = (21 * L + 255) // 256 * 256
    Npad = (N + 255) // 256 * 256
    nsp = 20 * L + 32 - (20 * L) % 32
    W = x[nsp:].reshape(Q, L, QP, L)[:, :, :Q, :]                       # [b,k,a,j] float32

    # compressed operand and metadata -> logical one-hot in the order l * 21 + q
    ac = fetch(ev, 9, np.uint8)[sp_a_index(Npad, KP)].astype(np.int64)
    meta = fetch(ev, 10, np.uint8)[sp_e_index(Npad, KP)].astype(np.int64)
    nib = np.stack([meta & 15, meta >> 4], axis=2).reshape(Npad, KP // 4)
    i0, i1 = nib & 3, nib >> 2
    assert np.all(i0 < i1)
    for idx, size in ((sp_a_index(Npad, KP), Npad * KP // 2), (sp_e_index(Npad, KP), Npad * KP // 8),
                      (sp_b_index(KP, SW), KP * SW)):
        assert idx.size == size and np.array_equal(np.sort(idx.ravel()), np.arange(size))
    logical = np.zeros((Npad, KP // 4, 4), dtype=np.int64)
    rows = np.arange(Npad)[:, None]
    grp = np.arange(KP // 4)[None, :]
    logical[rows, grp, i0] = ac[:, 0::2]
    logical[rows, grp, i1] += ac[:, 1::2]
    onehot_nat = np.zeros((Npad, KP), dtype=np.int64)
    for l in range(L):
        onehot_nat[np.arange(N), l * Q + msa[:, l].astype(np.int64)] = 1
    assert np.array_equal(logical.reshape(Npad, KP), onehot_nat)

    # one-hot of the backward in 192-slot groups, ones slot 189, read through the
    # backward's tiled storage
    bwd = sp_bwd_index(Npad, S)
    assert np.array_equal(np.sort(bwd.ravel()), np.arange(Npad * S))
    O1 = fetch(ev, 0, np.uint8)[bwd]
    O = np.zeros((Npad, S), dtype=np.uint8)
    for n in range(N):
        for l in range(L):
            O[n, slot192(int(msa[n, l]), l)] = 1
        O[n, 189] = 1
    assert np.array_equal(O1, O)

    # digits of W: rows k * 21 + b, columns s192(a, j), exact
    cm = fetch(ev, 8, np.uint32).view(np.float32).reshape(Q, L)
    mant, ex = np.frexp(cm.astype(np.float64))
    e = np.where(cm == 0, 0, np.where(mant == 0.5, ex - 1, ex))
    scale = np.ldexp(1.0, 21 - e)
    Wq = np.clip(np.rint(W.astype(np.float64) * scale[None, None]), -2**21, 2**21 - 1)
    bidx = sp_b_index(KP, SW)
    d = [fetch(ev, 1 + i, np.uint8)[bidx] for i in range(3)]
    Qgpu = digits_value(*d)
    Qexp = np.zeros((KP, SW), dtype=np.int64)
    rows_k = (np.arange(L)[None, :] * Q + np.arange(Q)[:, None]).reshape(-1)       # [b,k] -> k*21+b
    cols_s = np.array([[slot192(a, j) for j in range(L)] for a in range(Q)]).reshape(-1)
    Qexp[np.ix_(rows_k, cols_s)] = Wq.astype(np.int64).reshape(Q * L, Q * L)
    assert np.array_equal(Qgpu, Qexp)

    # R digits in 192-slot groups against the FP64 forward at the quantised W
    V = x[:20 * L].reshape(20, L).astype(np.float64)
    Wdeq = (Wq / scale[None, None]).reshape(Q * L, Q * L)               # rows (b,k), cols (a,j)
    Onat = np.zeros((N, Q * L))
    for l in range(L):
        Onat[np.arange(N), msa[:, l].astype(np.int64) * L + l] = 1.0    # column b*L + k
    logits = (Onat @ Wdeq).reshape(N, Q, L)                             # [n, a, j]
    r = [fetch(ev, 4 + i, np.uint8)[bwd] for i in range(3)]
    R_gpu = digits_value(*r) / 2.0**21
    R_exp = np.zeros((Npad, S))
    for l in range(L):
        z = logits[:, :, l].copy()
        z[:, :20] += V[:, l][None, :]
        z -= z.max(axis=1, keepdims=True)
        P = np.exp(z) / np.exp(z).sum(axis=1, keepdims=True)
        onehot = (msa[:, l][:, None] == np.arange(Q)[None, :]).astype(np.float64)
        R_exp[:N, [slot192(a, l) for a in range(Q)]] = w[:, None] * (P - onehot)
    assert np.abs(R_gpu - R_exp).max() < 2.0**-21 + 2e-6
    ev.close()
