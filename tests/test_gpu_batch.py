"""Batched solves (ccm_solve_batch): every alignment's result equals that of a
standalone solve of the same alignment (contexts are independent and each
solve is deterministic), whatever the number of concurrent workers."""
import numpy as np
import pytest

from ccmpred_b200 import _lib, solve_batch, synth

pytestmark = pytest.mark.gpu


def test_batch_matches_standalone_solves(gpu):
    msas = synth.batch_workload(10, seed0=500)
    msas = [m[: min(len(m), 1500)] for m in msas]          # keep the test short
    res4, maps4 = solve_batch(msas, workers=4, max_iterations=40)
    res1, maps1 = solve_batch(msas, workers=1, max_iterations=40)
    for r4, r1, m4, m1 in zip(res4, res1, maps4, maps1):
        assert r4.status in (_lib.CG_SUCCESS, _lib.CG_ERR_MAXITER)
        assert r4.iterations == r1.iterations and r4.fx == r1.fx
        assert np.array_equal(m4, m1)
        assert np.all(np.isfinite(m4))


def test_batch_rejects_bad_input(gpu):
    with pytest.raises(_lib.CcmError):
        solve_batch([np.zeros((5, 0), dtype=np.uint8)])
