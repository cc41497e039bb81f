"""Autotuner of the batched solver: per (L, N) bucket, the evaluation path --
and with it the tile shapes -- that gives the most evaluations per second when
several alignments of that size run at once.

The paths differ in how an alignment maps onto the tensor cores:

* ``tc_i8sp``: 256-row x 192-slot forward tiles (9 alignment columns), 2:4-sparse
  8-bit MMAs; 256 x 256 backward tiles over 192-slot groups;
* ``tc_i8x3``: 256 x 256 dense 8-bit tiles (12 columns per tile);
* ``tc_bf16x2``: 256 x 256 bf16 tiles, two split terms;
* ``simt_f32``: no tensor cores (CUDA-core kernels, no tile padding).

Small alignments fill few tiles and pay for the slot padding of a tile, so the
best choice depends on (L, N).  ``tune()`` times, for every bucket, ``streams``
contexts of that size evaluating concurrently on their own streams (the way a
wave of the batch solver runs them) and records evaluations per second per
path; ``choose()`` maps an alignment to the bucket that covers it.  Run on the
target GPU:

    python -m ccmpred_b200.autotune            # writes ccmpred_b200/tuning_b200.json

``solve_batch(..., path="auto")`` reads the table.
"""
from __future__ import annotations

import json
import os
import time
from typing import Dict, List, Optional

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
TABLE = os.path.join(HERE, "tuning_b200.json")

BUCKETS_L = [60, 120, 200, 300, 400]
BUCKETS_N = [300, 1000, 3000, 10000, 20000]
PATHS = ["tc_i8sp", "tc_i8x3", "tc_bf16x2", "simt_f32"]


def measure(L: int, N: int, path: str, streams: int = 4, budget_s: float = 1.0,
            device: int = 0) -> float:
    """Aggregate evaluations per second of `streams` contexts of an L x N synthetic
    alignment evaluating concurrently (CUDA events on each context's stream)."""
    import torch

    from . import Evaluator, _lib, synth
    msa = synth.generate(synth.MSAConfig("tune", L, N, n_pairs=min(4, L // 2), seed=L * 7 + N))
    evs, xs, gs = [], [], []
    try:
        for k in range(streams):
            ev = Evaluator(msa, path=path, device=device)
            x = torch.from_numpy(synth.random_x(L, 11 + k)).cuda(device)
            evs.append(ev)
            xs.append(x)
            gs.append(torch.empty_like(x))
        lib = _lib.lib()
        for ev, x, g in zip(evs, xs, gs):
            ev.evaluate(x, g)                      # warm-up
        torch.cuda.synchronize(device)
        # repetitions from one timed evaluation, bounded by the budget
        t0 = time.perf_counter()
        evs[0].evaluate(xs[0], gs[0])
        one = max(time.perf_counter() - t0, 1e-5)
        reps = int(max(2, min(50, budget_s / (one * streams))))
        starts, ends = [], []
        for ev in evs:
            st = torch.cuda.ExternalStream(ev.stream, device=torch.device("cuda", device))
            a = torch.cuda.Event(enable_timing=True)
            a.record(st)
            starts.append((a, st))
        for _ in range(reps):
            for ev, x, g in zip(evs, xs, gs):
                _lib.check(lib.ccm_evaluate_async(ev.handle, x.data_ptr(), g.data_ptr(), x.numel()))
        for a, st in starts:
            b = torch.cuda.Event(enable_timing=True)
            b.record(st)
            ends.append(b)
        torch.cuda.synchronize(device)
        # the concurrent span: earliest start to latest end
        t_ms = max(starts[0][0].elapsed_time(b) for b in ends)
        return streams * reps / (t_ms / 1e3)
    finally:
        for ev in evs:
            ev.close()


def tune(buckets_L: List[int] = BUCKETS_L, buckets_N: List[int] = BUCKETS_N,
         paths: List[str] = PATHS, streams: int = 4, device: int = 0) -> Dict:
    import torch
    rows = []
    for L in buckets_L:
        for N in buckets_N:
            evals = {}
            for path in paths:
                try:
                    evals[path] = measure(L, N, path, streams=streams, device=device)
                except Exception as exc:           # a path that cannot run this size
                    evals[path] = None
                    print(f"autotune: L={L} N={N} {path}: {exc}")
            ok = {p: v for p, v in evals.items() if v}
            best = max(ok, key=ok.get)
            rows.append({"L": L, "N": N, "path": best, "evals_per_s": evals})
            print(f"autotune: L={L:4d} N={N:6d} -> {best:10s} "
                  + " ".join(f"{p}={v:.0f}" for p, v in ok.items()))
    return {"device": torch.cuda.get_device_name(device), "streams": streams,
            "metric": "aggregate evaluations/s of concurrent contexts of the bucket's size",
            "buckets_L": buckets_L, "buckets_N": buckets_N, "rows": rows}


def load(path: str = TABLE) -> Optional[Dict]:
    if not os.path.exists(path):
        return None
    with open(path) as f:
        return json.load(f)


def choose(table: Dict, L: int, N: int) -> str:
    """The path of the smallest bucket with L_b >= L and N_b >= N (the largest
    bucket beyond the table's range)."""
    bl = next((b for b in table["buckets_L"] if b >= L), table["buckets_L"][-1])
    bn = next((b for b in table["buckets_N"] if b >= N), table["buckets_N"][-1])
    for r in table["rows"]:
        if r["L"] == bl and r["N"] == bn:
            return r["path"]
    return "tc_i8sp"


def main():
    import sys
    out = sys.argv[1] if len(sys.argv) > 1 else TABLE
    table = tune()
    with open(out, "w") as f:
        json.dump(table, f, indent=1)
    print(f"wrote {out}")


if __name__ == "__main__":
    main()
