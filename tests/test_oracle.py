"""The oracle is pinned: FP64 restatement and reweighting vs the reference's own
compiled code and vs the committed golden vectors (CPU only)."""
import glob
import os

import numpy as np
import pytest

from ccmpred_b200 import synth

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def rel(a, b):
    return float(np.linalg.norm(np.asarray(a, np.float64) - b) / max(np.linalg.norm(b), 1e-300))


@pytest.mark.parametrize("path", sorted(glob.glob(os.path.join(GOLDEN, "eval_*.npz"))))
def test_oracle_matches_golden_evaluate(oracle_mod, path):
    d = np.load(path)
    f64, g64 = oracle_mod.oracle_evaluate(d["msa"], d["weights"], float(d["lambda_single"]),
                                          float(d["lambda_pair"]), d["x"])
    # the golden f/g come from the reference's FP32 evaluate_cpu: agreement at FP32 level
    assert abs(float(d["f"]) - f64) / abs(f64) < 2e-6
    assert rel(d["g"], g64) < 2e-6


def test_oracle_weights_match_golden(oracle_mod):
    d = np.load(os.path.join(GOLDEN, "weights_L40_N300_dup.npz"))
    for t in d["thresholds"]:
        w = oracle_mod.oracle_weights(d["msa"], float(t))
        ref = d[f"w_{int(round(float(t) * 100))}"]
        assert np.array_equal(w.view(np.uint32), ref.view(np.uint32)), t


@pytest.mark.parametrize("L,N,seed,xkind", [(3, 5, 1, "rand"), (12, 40, 2, "bias"),
                                            (13, 64, 3, "rand"), (25, 120, 4, "rand"),
                                            (1, 7, 5, "rand")])
def test_oracle_matches_reference_evaluate(ref_mod, L, N, seed, xkind):
    msa = synth.generate(synth.MSAConfig("t", L, N, n_pairs=min(2, L // 2), dup_frac=0.2, seed=seed))
    lam1, lam2 = 0.01, 0.2 * max(L - 1, 1)
    ev = ref_mod.RefEvaluator(msa, lam1, lam2, 0.8)
    x = ref_mod.ref_init_bias(msa) if xkind == "bias" else synth.random_x(L, seed)
    f, g = ev.evaluate(x)
    w = ev.weights
    ev.close()
    f64, g64 = ref_mod.oracle_evaluate(msa, w, lam1, lam2, x)
    assert abs(f - f64) / abs(f64) < 2e-6
    assert rel(g, g64) < 2e-6


def test_oracle_inadmissible_x_matches_reference(ref_mod):
    """Non-zero padding and self blocks: the CPU reference semantics (2*lambda2*x
    on self blocks and padding, g1 padding 0) are restated exactly."""
    L, N = 7, 30
    msa = synth.generate(synth.MSAConfig("t", L, N, seed=9))
    rng = np.random.default_rng(0)
    x = rng.normal(0, 0.05, ref_mod.nvar_padded(L)).astype(np.float32)
    ev = ref_mod.RefEvaluator(msa, 0.01, 1.2, 0.8)
    f, g = ev.evaluate(x)
    w = ev.weights
    ev.close()
    f64, g64 = ref_mod.oracle_evaluate(msa, w, 0.01, 1.2, x)
    assert abs(f - f64) / abs(f64) < 2e-6
    assert rel(g, g64) < 2e-6


@pytest.mark.parametrize("thr", [0.5, 0.8, 0.9, 1.0])
def test_oracle_weights_bit_exact_vs_reference(ref_mod, thr):
    msa = synth.generate(synth.MSAConfig("t", 33, 257, gap_frac=0.2, dup_frac=0.5, seed=7))
    a = ref_mod.oracle_weights(msa, thr)
    b = ref_mod.ref_calculate_weights(msa, thr)
    assert np.array_equal(a.view(np.uint32), b.view(np.uint32))


def test_oracle_weights_on_example_alignment(ref_mod):
    path = ref_mod.REF_EXAMPLE_ALN
    if not os.path.exists(path):
        pytest.skip("reference example alignment not copied into oracle/_ref")
    msa = ref_mod.ref_read_msa(path)
    assert msa.shape == (3068, 75)
    a = ref_mod.oracle_weights(msa, 0.8)
    b = ref_mod.ref_calculate_weights(msa, 0.8)
    assert np.array_equal(a.view(np.uint32), b.view(np.uint32))


def test_synthetic_generator_is_seeded():
    a = synth.generate(synth.SMALL_75x1000)
    b = synth.generate(synth.SMALL_75x1000)
    assert a.shape == (1000, 75) and a.dtype == np.uint8
    assert np.array_equal(a, b)
    assert a.max() <= 20
    gap = (a == 20).mean()
    assert 0.05 < gap < 0.2
    x = synth.random_x(9, 3)
    L = 9
    nsp = 180 + 32 - 180 % 32
    W = x[nsp:].reshape(21, L, 32, L)
    assert np.allclose(W[:, :, :21, :], np.transpose(W[:, :, :21, :], (2, 3, 0, 1)))
    assert np.all(W[:, :, 21:, :] == 0)
    for k in range(L):
        assert np.all(W[:, k, :, k] == 0)
