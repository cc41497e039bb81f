"""Generate the golden vectors in tests/golden/ from the reference's own code.

Run where the reference checkout exists (it builds oracle/_ref/libccmref.so
from the reference sources via oracle/Makefile):

    python tests/golden/make_golden.py

Every array is produced by the reference's compiled C functions
(evaluate_cpu, calculate_weights, init_bias, sum_submatrices, apc) on seeded
synthetic inputs, so the fixtures pin the oracle and the CUDA path to the
reference's behaviour without the reference being present at test time.
"""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from ccmpred_b200 import synth  # noqa: E402
from oracle import oracle as O  # noqa: E402

OUT = os.path.dirname(os.path.abspath(__file__))


def evaluate_case(name, cfg, x_kind, thr=0.8):
    msa = synth.generate(cfg)
    N, L = msa.shape
    lam1, lam2 = 0.01, 0.2 * (L - 1)
    ev = O.RefEvaluator(msa, lam1, lam2, thr)
    if x_kind == "bias":
        x = O.ref_init_bias(msa)
    else:
        x = synth.random_x(L, seed=cfg.seed + 100)
    f, g = ev.evaluate(x)
    w = ev.weights
    ev.close()
    cmap = O.ref_contact_map(x, L, apc=True)
    np.savez_compressed(os.path.join(OUT, f"{name}.npz"), msa=msa, x=x, weights=w, f=np.float32(f),
                        g=g, lambda_single=np.float32(lam1), lambda_pair=np.float32(lam2),
                        threshold=np.float32(thr), contact_map_apc=cmap)
    print(name, msa.shape, f)


def weights_case(name, cfg, thresholds):
    msa = synth.generate(cfg)
    ws = {f"w_{int(round(t * 100))}": O.ref_calculate_weights(msa, t) for t in thresholds}
    np.savez_compressed(os.path.join(OUT, f"{name}.npz"), msa=msa,
                        thresholds=np.array(thresholds, dtype=np.float32), **ws)
    print(name, msa.shape, {k: float(v.sum()) for k, v in ws.items()})


if __name__ == "__main__":
    O.build()
    evaluate_case("eval_L9_N31_bias", synth.MSAConfig("g1", 9, 31, n_pairs=2, seed=21), "bias")
    evaluate_case("eval_L9_N31_rand", synth.MSAConfig("g2", 9, 31, n_pairs=2, seed=22), "rand")
    evaluate_case("eval_L14_N45_rand", synth.MSAConfig("g3", 14, 45, n_pairs=3, dup_frac=0.3,
                                                       seed=23), "rand", thr=0.7)
    weights_case("weights_L40_N300_dup", synth.MSAConfig("g4", 40, 300, gap_frac=0.2,
                                                          dup_frac=0.4, seed=24),
                 [0.5, 0.62, 0.8, 0.9])
