#!/usr/bin/env python
"""Benchmark: pseudo-likelihood + gradient evaluations per second at L=300, N=5000.

One step = one evaluation of f and the full gradient at a fixed parameter
vector x (the reference's evaluate callback, src/evaluate_cuda.c:23-74),
through the C ABI of libccmpred_b200.so.

  value       evals/s of the default path (--path, tc_i8sp: 8-bit fixed-point
              digits with exact integer sums on the tensor cores) with x and g
              resident in HBM (ccm_evaluate_async back to back, CUDA events on
              the context stream, max over ranks); the split-bf16 path the
              metric names is timed beside it (tc_bf16x2);
  e2e         evals/s through the host-pointer C ABI (ccm_evaluate_host):
              every step copies x host->device from pinned memory and g + f
              device->host;
  roofline    the dominant tcgen05 GEMM kernel, algorithmic FLOPs per launch
              (2 N (21 L)^2, counted once: no hi/lo doubling, no padding) over
              its CUDA-event time inside the timed region;
  plain_f32   the same metric on the plain FP32 CUDA-core path (no tensor cores);
  precision   errors of f and g against the FP64 oracle at the same x;
  cpu_baseline the reference's evaluate_cpu_omp (compiled from its sources)
              on a bounded sample, on this host's cores;
  batch256, L1000_N20000  (N=1, after the timed region; --no-extras skips them)
              the lines of --workload batch256 and --workload L1000_N20000.

`--impl reference` times the reference's own CPU implementation
(evaluate_cpu_omp, all host threads) on the same workload instead.
Multi-GPU (torchrun): replicas only -- every rank evaluates its own copy of
the workload; no data-path collective exists for a single alignment.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "PLL+grad evals/s at L=300 N=5000: split-BF16 TC vs plain FP32, rel err≤1e-5"
UNIT = "evals/s"
WORKLOAD = "L300_N5000"
REF_BUDGET_S = 120.0  # bound of the reference arm's timed loop (CPU, ~1 s per evaluation)



PATH_DTYPE = {"tc_bf16x2": "bf16", "tc_bf16x3": "bf16", "tc_i8x3": "int8", "tc_i8sp": "int8"}
PATH_ARITHMETIC = {
    "tc_bf16x2": "bf16 hi+lo split operands, f32 tensor-core accumulation, "
                 "f64 loss/regulariser reductions",
    "tc_bf16x3": "three bf16 terms per operand, f32 tensor-core accumulation, "
                 "f64 loss/regulariser reductions",
    "tc_i8x3": "W and R as three 8-bit fixed-point digits (21 fractional bits, per-column "
               "power-of-two scale for W), exact s32 tensor-core accumulation, "
               "f64 loss/regulariser reductions",
    "tc_i8sp": "as tc_i8x3 (the same exact integer sums), with the forward on 2:4-sparse "
               "tcgen05.mma.sp over the compressed one-hot operand",
}


_JSON_FD = None


def quiet_stdout():
    """Route everything written to stdout -- Python's prints and the C libraries'
    printf (the reference's init prints its reweighting summary) -- to stderr, so
    that the original stdout carries exactly the one JSON line (see emit)."""
    global _JSON_FD
    sys.stdout.flush()
    _JSON_FD = os.dup(1)
    os.dup2(2, 1)


def emit(obj):
    fd = _JSON_FD if _JSON_FD is not None else 1
    os.write(fd, (json.dumps(obj) + "\n").encode())

def parse_args():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=1000)
    p.add_argument("--warmup", type=int, default=10)
    p.add_argument("--impl", default="b200", choices=["b200", "reference"])
    p.add_argument("--path", default="tc_i8sp",
                   choices=["tc_i8sp", "tc_i8x3", "tc_bf16x2", "tc_bf16x3"])
    p.add_argument("--e2e-steps", type=int, default=50)
    p.add_argument("--plain-steps", type=int, default=20)
    p.add_argument("--compare-steps", type=int, default=300,
                   help="evaluations of the split-bf16 path timed beside the default path")
    p.add_argument("--cpu-budget-s", type=float, default=15.0)
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--no-precision", action="store_true")
    p.add_argument("--workload", default="L300_N5000",
                   choices=["L300_N5000", "L1000_N20000", "batch256"],
                   help="L1000_N20000: 100 CG iterations on the large alignment as one "
                        "device-side solve (ms/iteration, evals/s); batch256: 256 ragged "
                        "alignments solved to convergence (MSAs/s)")
    p.add_argument("--cg-iterations", type=int, default=100)
    p.add_argument("--batch-workers", type=int, default=8)
    p.add_argument("--batch-plain-sample", type=int, default=8)
    p.add_argument("--no-extras", action="store_true",
                   help="leave the batch256 and L1000_N20000 results out of the default line "
                        "(N=1 only; they run after the headline's timed region)")
    p.add_argument("--ref-cuda-steps", type=int, default=3,
                   help="evaluations of the reference's own CUDA kernels (sm_100a build); 0 = skip")
    return p.parse_args()


def workload():
    from ccmpred_b200 import synth
    cfg = synth.PRECISION_300x5000
    msa = synth.generate(cfg)
    x = synth.random_x(cfg.ncol, seed=cfg.seed + 1000)
    return cfg, msa, x


def workload_config(cfg, world):
    """The `config` of both arms: what identifies the workload, nothing about
    the implementation that runs it."""
    return {"workload": WORKLOAD, "ncol": cfg.ncol, "nrow": cfg.nrow,
            "planted_pairs": cfg.n_pairs, "seed": cfg.seed,
            "l2": "inputs larger than L2 (x and g 242 MB each)",
            "parallelism": f"replicas x{world}"}


def measured_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            d = json.load(f)
        return d, "measured"
    return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "bf16_tflops_sustained": 1400.0}, "fallback"


def tensor_peak(peaks, peak_kind, clocks, elapsed_ms):
    """The bf16 denominator for a tensor-bound kernel: the burst figure (measured at
    the maximum SM clock) or the sustained one (measured under the power cap, at the
    lower clock recorded beside it), whichever was taken at the clock nearer the
    median SM clock this timed region held.  Without clock samples, the length of
    the timed region decides (a region under a second keeps the maximum clock).
    Returns (peak, name, why)."""
    burst = float(peaks.get("bf16_tflops", peaks.get("bf16_tflops_sustained")))
    sustained = float(peaks.get("bf16_tflops_sustained", burst))
    f_burst = float(peaks.get("sm_max_mhz") or 1965.0)
    f_sus = (peaks.get("clocks_under_load") or {}).get("sm_mhz_median")
    held = (clocks or {}).get("sm_mhz")
    if held and f_sus:
        mid = 0.5 * (f_burst + float(f_sus))
        if held >= mid:
            peak, name = burst, "bf16_tflops"
            why = f"burst: median SM clock {held:.0f} MHz, nearer {f_burst:.0f} than {f_sus:.0f}"
        else:
            peak, name = sustained, "bf16_tflops_sustained"
            why = f"sustained: median SM clock {held:.0f} MHz, nearer {f_sus:.0f} than {f_burst:.0f}"
    elif elapsed_ms < 1000.0:
        peak, name = burst, "bf16_tflops"
        why = f"burst: timed region {elapsed_ms:.0f} ms < 1 s, no clock samples"
    else:
        peak, name = sustained, "bf16_tflops_sustained"
        why = f"sustained: timed region {elapsed_ms:.0f} ms >= 1 s, no clock samples"
    if peak_kind == "fallback":
        why += "; MEASURED_PEAKS.json absent"
    return peak, name, why


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.tmp = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200", "-i", str(self.index)], stdout=self.tmp, stderr=subprocess.DEVNULL)
        except (FileNotFoundError, OSError):
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.tmp.flush()
        self.tmp.seek(0)
        rows = [r.strip().split(",") for r in self.tmp.read().splitlines() if r.strip()]
        os.unlink(self.tmp.name)
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            r = [c.strip() for c in r]
            if len(r) < 9:
                continue
            try:
                sm.append(float(r[1]))
                mx = float(r[2])
            except ValueError:
                continue
            for name, val in zip(names, r[5:9]):
                if val.lower().startswith("active"):
                    reasons.add(name)
        if not sm:
            return None
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def dist_init(args=None, backend: str = "nccl"):
    """One process per GPU (torchrun env).  NCCL carries only the barrier and the
    max-over-ranks timing: the workload is replicated, nothing is exchanged."""
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist
        if backend == "nccl":
            torch.cuda.set_device(local)
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=120))
    return world, rank, local


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def max_over_ranks(world, value: float) -> float:
    if world == 1:
        return value
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([value], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def cpu_reference_timing(msa, x, budget_s, max_evals, omp=True):
    """Reference evaluate_cpu_omp (all host threads), or with omp=False the serial
    evaluate_cpu: (evals/s, evaluations, kind, cores)."""
    from oracle import oracle as O
    N, L = msa.shape
    cores = (os.cpu_count() or 1) if omp else 1
    if O.ref_available():
        ev = O.RefEvaluator(msa, 0.01, 0.2 * (L - 1), 0.8, omp=omp)
        times = []
        t_start = time.perf_counter()
        try:
            for _ in range(max_evals):
                t0 = time.perf_counter()
                ev.evaluate(x)
                times.append(time.perf_counter() - t0)
                if time.perf_counter() - t_start > budget_s:
                    break
        finally:
            ev.close()
        return 1.0 / float(np.median(times)), len(times), "reference", cores
    w = O.oracle_weights(msa, 0.8)
    times = []
    t_start = time.perf_counter()
    for _ in range(max_evals):
        t0 = time.perf_counter()
        O.oracle_evaluate(msa, w, 0.01, 0.2 * (L - 1), x)
        times.append(time.perf_counter() - t0)
        if time.perf_counter() - t_start > budget_s:
            break
    return 1.0 / float(np.median(times)), len(times), "port", cores


def run_reference_arm(args, world, rank):
    if rank != 0:
        return
    from oracle import oracle as O
    cfg, msa, x = workload()
    if not O.ref_available():
        emit(({"impl": "reference", "unavailable":
                          "oracle/_ref/libccmref.so (reference CPU sources) was not built"}))
        return
    N, L = msa.shape
    ev = O.RefEvaluator(msa, 0.01, 0.2 * (L - 1), 0.8, omp=True)
    # one evaluation takes about a second on 16 host cores: the warm-up and the timed
    # steps are bounded samples (at most 3 warm-up evaluations, and the timed loop
    # stops after the first evaluation that ends past REF_BUDGET_S), so that the
    # default --steps still finishes within a few minutes
    for _ in range(min(args.warmup, 3)):
        ev.evaluate(x)
    t0 = time.perf_counter()
    timed = 0
    while timed < args.steps:
        ev.evaluate(x)
        timed += 1
        if time.perf_counter() - t0 > REF_BUDGET_S:
            break
    el = time.perf_counter() - t0
    ev.close()
    value = timed / el
    cores = os.cpu_count() or 1
    emit(({
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "steps_timed": timed, "warmup": args.warmup,
        "warmup_run": min(args.warmup, 3),
        "ms_per_step": el / timed * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic",
        "config": workload_config(cfg, world),
        "impl_detail": "reference evaluate_cpu_omp.c compiled from its sources (-O3 -fopenmp), "
                       "all host threads",
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "reference",
                         "sample": f"{timed} full evaluations at L=300 N=5000 (of the "
                                   f"{args.steps} steps asked; at most {REF_BUDGET_S:.0f} s)"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }))


def precision_block(msa, w, x, g_gpu, f_gpu, L):
    from ccmpred_b200 import nsingle_padded
    from oracle import oracle as O
    # lambda2 as the evaluators compute it (the reference's float 0.2f * (L - 1))
    f64, g64 = O.oracle_evaluate(msa, w, 0.01, float(np.float32(0.2) * np.float32(L - 1)), x)
    d = g_gpu.astype(np.float64) - g64
    nsp, ns = nsingle_padded(L), 20 * L
    n = np.linalg.norm
    return {"f_rel": abs(f_gpu - f64) / abs(f64), "g_rel": float(n(d) / n(g64)),
            "g1_rel": float(n(d[:ns]) / n(g64[:ns])), "g2_rel": float(n(d[nsp:]) / n(g64[nsp:])),
            "reference": "FP64 oracle (oracle/ccm_oracle.c) at the same x and weights"}


def reference_cuda_timing(msa, x, xd, steps, with_precision):
    """The reference's own CUDA evaluator (evaluate_cuda.c + evaluate_cuda_kernels.cu built
    for sm_100a from its sources), same x, device pointers, host-synchronised like the
    reference (it returns f by value and syncs after every kernel)."""
    import torch
    from oracle import oracle as O
    if not os.path.exists(O.REF_CUDA_SO):
        return {"unavailable": "oracle/_ref/libccmref_cuda.so was not built"}
    N, L = msa.shape
    ev = O.RefCudaEvaluator(msa, 0.01, 0.2 * (L - 1), 0.8)
    g = torch.empty_like(xd)
    f = ev.evaluate(xd.data_ptr(), g.data_ptr())
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(steps):
        ev.evaluate(xd.data_ptr(), g.data_ptr())
    torch.cuda.synchronize()
    el = time.perf_counter() - t0
    out = {"evals_per_s": steps / el, "steps": steps,
           "impl": "reference evaluate_cuda + evaluate_cuda_kernels.cu compiled for sm_100a "
                   "(SIMT FP32, fdexp/fdlog = expf/logf)"}
    if with_precision:
        w = O.ref_calculate_weights(msa, 0.8)
        out["precision"] = precision_block(msa, w, x, g.cpu().numpy(), f, L)
    ev.close()
    return out


def traffic_from_profiles(kernel: str, path_name: str):
    """DRAM bytes per launch of the dominant kernel from the committed ncu summary
    of the path's kernels (tc_* for the bf16 paths, i8_* for the integer path)."""
    if path_name == "tc_i8sp":
        fname = "i8sp_kernels_L300_N5000.json"
        kernel = {"tc_forward": "i8sp_forward"}.get(kernel, kernel.replace("tc_", "i8_"))
    elif path_name == "tc_i8x3":
        fname, kernel = "i8_kernels_L300_N5000.json", kernel.replace("tc_", "i8_")
    else:
        fname = "tc_kernels_L300_N5000.json"
    path = os.path.join(ROOT, "profiles", fname)
    if not os.path.exists(path):
        return None
    with open(path) as f:
        d = json.load(f)
    k = d.get("kernels", {}).get(kernel)
    return None if k is None else k.get("dram_bytes_per_launch")


def run_batch(args, world, rank, local, emit_line=True):
    """256 ragged alignments (L ~ U[50,400], N ~ logU[200,20000]) solved to convergence
    (eps 1e-3 or 250 iterations) concurrently, vs one at a time on the plain FP32 path
    (timed on a stratified sample and extrapolated).  Returns the line (rank 0)."""
    import torch
    import ccmpred_b200 as cb
    from ccmpred_b200 import synth
    torch.cuda.set_device(local)
    from ccmpred_b200 import autotune
    msas = synth.batch_workload(256, seed0=1000 + 1000 * rank)
    cb.solve_batch(msas[:2], workers=2, max_iterations=3, epsilon=1e-3, device=local)  # warm-up
    torch.cuda.synchronize()
    # the headline: solve_batch's defaults (host worker threads, each running whole
    # device-side solves, one path for all); beside it each alignment's path from
    # the autotuner's table, and waves (one graph launch per wave of alignments)
    runs = [("threads", args.path), ("threads", "auto" if autotune.load() else args.path),
            ("waves", args.path)]
    if runs[0] == runs[1]:
        runs = runs[1:]
    timed = {}
    res = None
    for mode, path in runs:
        barrier(world)
        t0 = time.perf_counter()
        r, _ = cb.solve_batch(msas, workers=args.batch_workers, path=path, max_iterations=250,
                              epsilon=1e-3, device=local, waves=(mode == "waves"))
        torch.cuda.synchronize()
        el_r = max_over_ranks(world, time.perf_counter() - t0)
        timed[f"{mode}/{path}"] = {"msas_per_s": world * len(msas) / el_r, "wall_s": el_r,
                                   "iterations_mean": float(np.mean([x.iterations for x in r]))}
        if res is None:
            res, el = r, el_r
    value = world * len(msas) / el
    if rank != 0:
        return None
    cost = np.array([m.shape[0] * m.shape[1] ** 2 for m in msas], dtype=np.float64)
    order = np.argsort(cost)
    k = args.batch_plain_sample
    sample = [int(order[int((i + 0.5) * len(order) / k)]) for i in range(k)]
    plain_t = []
    for i in sample:
        t1 = time.perf_counter()
        cb.solve_batch([msas[i]], workers=1, path="simt_f32", max_iterations=250, epsilon=1e-3,
                       device=local)
        plain_t.append(time.perf_counter() - t1)
    plain_total = float(np.sum(plain_t) * len(msas) / k)
    its = np.array([r.iterations for r in res])
    ok = sum(r.status in (0, -1023) for r in res)
    line = {
        "metric": "MSAs/s, 256 ragged alignments solved to convergence", "value": value,
        "unit": "MSAs/s", "n_gpus": world, "higher_is_better": True, "scaling": "weak",
        "data": "synthetic", "dtype": "int8",
        "config": {"workload": "batch256: L~U[50,400], N~logU[200,20000], seeds 1000+i, "
                               "eps 1e-3 or 250 iterations",
                   "mode": f"{runs[0][0]}/{runs[0][1]}"},
        "wall_s": el, "solved_ok": ok, "iterations_mean": float(its.mean()),
        "by_mode": timed,
        "plain_f32_one_at_a_time": {
            "msas_per_s_extrapolated": len(msas) / plain_total,
            "sample": f"{k} alignments stratified by N*L^2, timed one at a time, "
                      f"scaled to {len(msas)}",
            "speedup": value / (len(msas) / plain_total)},
    }
    if emit_line:
        emit(line)
    return line


def run_large(args, world, rank, local, emit_line=True, with_cpu=True):
    """L=1000, N=20000 (20 % gaps, 30 % near-duplicate rows): GPU reweighting,
    init_bias, then --cg-iterations CG iterations as ONE device-side solve (line
    search, direction update and iteration loop in a CUDA graph with conditional
    nodes; the host waits once), timed with CUDA events on the context stream.
    The gradient at the final x is checked against the FP64 CUDA-core path.
    Returns the line (rank 0); with_cpu=False leaves out the reference CPU sample
    (one evaluation, about 40 s)."""
    import ctypes

    import torch

    import ccmpred_b200 as cb
    from ccmpred_b200 import _lib, synth
    from ccmpred_b200.host import init_bias
    torch.cuda.set_device(local)
    cfg = synth.LARGE_1000x20000
    msa = synth.generate(cfg)
    N, L = msa.shape
    t0 = time.perf_counter()
    w = cb.calculate_weights(msa, 0.8, device=local)
    weights_ms = (time.perf_counter() - t0) * 1e3
    lam2 = float(np.float32(0.2) * np.float32(L - 1))
    lib = _lib.lib()
    ev = cb.Evaluator(msa, weights=w, lambda_pair=lam2, path=args.path, device=local)
    stream = torch.cuda.ExternalStream(ev.stream, device=torch.device("cuda", local))
    x0 = torch.from_numpy(init_bias(msa)).cuda()
    g = torch.empty_like(x0)
    # warm-up: module load, graph construction, a short solve
    ev.minimize(x0.clone(), max_iterations=2, epsilon=0.0)
    # one evaluation's kernels (CUDA events per kernel)
    _lib.check(lib.ccm_profile_begin(ev.handle, 3))
    for _ in range(3):
        _lib.check(lib.ccm_evaluate_async(ev.handle, x0.data_ptr(), g.data_ptr(), x0.numel()))
    kms = (ctypes.c_double * 8)()
    nk, ne = ctypes.c_int(0), ctypes.c_int(0)
    _lib.check(lib.ccm_profile_end(ev.handle, kms, 8, ctypes.byref(nk), ctypes.byref(ne)))
    names = ["prep", "forward", "backward", "finalize"]
    kernels = {names[i]: kms[i] / max(ne.value, 1) for i in range(min(nk.value, 4))}
    f_x0 = ev.evaluate(x0, g)
    gnorm_x0 = float(torch.linalg.vector_norm(g.double()))
    torch.cuda.synchronize()
    xs = x0.clone()
    launches0 = lib.ccm_launch_count(ev.handle)
    sampler = ClockSampler(local)
    barrier(world)
    torch.cuda.synchronize()
    sampler.start()
    time.sleep(0.3)
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record(stream)
    res = ev.minimize(xs, max_iterations=args.cg_iterations, epsilon=0.0)
    b.record(stream)
    b.synchronize()
    clocks = sampler.stop()
    elapsed_ms = max_over_ranks(world, a.elapsed_time(b))
    launches = lib.ccm_launch_count(ev.handle) - launches0
    if rank != 0:
        ev.close()
        return None
    # the gradient at the final x against the FP64 CUDA-core path
    f_tc = ev.evaluate(xs, g)
    g_tc = g.double().cpu().numpy()
    ev.close()
    with cb.Evaluator(msa, weights=w, lambda_pair=lam2, path="simt_f64", device=local) as r64:
        g64 = torch.empty_like(xs, dtype=torch.float64)
        f64 = r64.evaluate(xs.double(), g64)
        g64 = g64.cpu().numpy()
    # the plain FP32 CUDA-core path at the same x, for scale: near a minimum g is
    # small and every FP32 evaluator's absolute error weighs more
    with cb.Evaluator(msa, weights=w, lambda_pair=lam2, path="simt_f32", device=local) as r32:
        f32 = r32.evaluate(xs, g)
        g32 = g.double().cpu().numpy()
    nrm = np.linalg.norm
    nsp = cb.nsingle_padded(L)

    def prec(fv, gv):
        d = gv - g64
        return {"f_rel": abs(fv - f64) / abs(f64), "g_rel": float(nrm(d) / nrm(g64)),
                "g1_rel_of_g": float(nrm(d[:20 * L]) / nrm(g64)),
                "g2_rel_of_g": float(nrm(d[nsp:]) / nrm(g64))}
    peaks, peak_kind = measured_peaks()
    peak, peak_name, peak_why = tensor_peak(peaks, peak_kind, clocks, elapsed_ms)
    flops_eval = 4.0 * N * (21 * L) ** 2
    achieved = flops_eval * res.evaluations / (elapsed_ms / 1e3) / 1e12
    its = max(res.iterations, 1)
    cpu = None
    if with_cpu and not args.no_cpu_baseline and world == 1:
        # one evaluation of the reference's evaluate_cpu_omp at the final x (about
        # half a minute on the host cores; x, g and its per-call scratch take ~11 GB),
        # in iterations/s at this solve's evaluations per iteration
        v, n_ev, kind, cores = cpu_reference_timing(msa, xs.cpu().numpy(), 0.0, 1)
        per_it = res.evaluations / its
        cpu = {"value": v / per_it, "unit": "iterations/s", "cores": cores, "kind": kind,
               "evals_per_s": v,
               "sample": f"{n_ev} full evaluation of the L=1000 N=20000 workload at the final x, "
                         f"evaluate_cpu_omp with all {cores} host threads; iterations/s at "
                         f"{per_it:.2f} evaluations per iteration (this solve's)"}
    line = {
        "metric": f"CG iterations/s at L=1000 N=20000 ({args.cg_iterations} iterations, one "
                  "device-side solve)",
        "value": res.iterations / (elapsed_ms / 1e3), "unit": "iterations/s", "n_gpus": world,
        "higher_is_better": True, "scaling": "weak", "data": "synthetic",
        "dtype": PATH_DTYPE[args.path],
        "config": {"workload": "L1000_N20000", "ncol": L, "nrow": N, "gap_frac": cfg.gap_frac,
                   "dup_frac": cfg.dup_frac, "seed": cfg.seed, "path": args.path,
                   "cg": f"{args.cg_iterations} iterations, epsilon 0 (no early stop), "
                         "max_linesearch 5, ftol 1e-4, wolfe 0.2 (float values)"},
        "ms_per_iteration": elapsed_ms / its, "solve_ms": elapsed_ms,
        "iterations": res.iterations, "evaluations": res.evaluations,
        "evals_per_s": res.evaluations / (elapsed_ms / 1e3), "cg_status": res.status,
        "kernels_ms_per_evaluation": kernels,
        "roofline": {"bound": "tensor", "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                     "frac": achieved / peak, "peak_source": f"{peak_kind} {peak_name} ({peak_why})",
                     "flops_per_evaluation": flops_eval,
                     "note": "useful FLOPs of both contractions per evaluation over the whole "
                             "solve's time (CG vector passes and graph overhead included)"},
        "objective": {"f_x0": f_x0, "gnorm_x0": gnorm_x0, "f_final": f64,
                      "gnorm_final": float(nrm(g64)),
                      "note": "f and ||g|| at x0 (this path) and at the final x (FP64 path)"},
        "precision_at_final_x": {
            args.path: prec(f_tc, g_tc), "simt_f32": prec(f32, g32),
            "reference": "FP64 CUDA-core path (simt_f64) at the same x"},
        "gpu_launches": int(launches), "clocks": clocks,
        "init_ms": {"weights": weights_ms},
        "cpu_baseline": cpu,
    }
    if emit_line:
        emit(line)
    return line


def main():
    args = parse_args()
    quiet_stdout()
    world, rank, local = dist_init(args)
    if args.impl == "b200" and args.workload == "batch256":
        run_batch(args, world, rank, local)
        barrier(world)
        return
    if args.impl == "b200" and args.workload == "L1000_N20000":
        run_large(args, world, rank, local)
        barrier(world)
        return
    if args.impl == "reference":
        run_reference_arm(args, world, rank)
        barrier(world)
        return

    import torch

    import ccmpred_b200 as cb
    from ccmpred_b200 import _lib

    torch.cuda.set_device(local)
    cfg, msa, x = workload()
    N, L = msa.shape
    t0 = time.perf_counter()
    w = cb.calculate_weights(msa, 0.8, device=local)
    init_ms = (time.perf_counter() - t0) * 1e3

    ev = cb.Evaluator(msa, weights=w, path=args.path, device=local)
    xd = torch.from_numpy(x).cuda()
    gd = torch.empty_like(xd)
    stream = torch.cuda.ExternalStream(ev.stream, device=torch.device("cuda", local))
    for _ in range(max(args.warmup, 3)):
        ev.evaluate(xd, gd)
    torch.cuda.synchronize()

    lib = _lib.lib()
    sampler = ClockSampler(local)
    launches0 = lib.ccm_launch_count(ev.handle)
    _lib.check(lib.ccm_profile_begin(ev.handle, args.steps))
    barrier(world)
    torch.cuda.synchronize()
    sampler.start()
    time.sleep(0.3)
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    start.record(stream)
    for _ in range(args.steps):
        _lib.check(lib.ccm_evaluate_async(ev.handle, xd.data_ptr(), gd.data_ptr(), xd.numel()))
    end.record(stream)
    end.synchronize()
    torch.cuda.synchronize()
    clocks = sampler.stop()
    barrier(world)
    elapsed_ms = start.elapsed_time(end)
    launches = lib.ccm_launch_count(ev.handle) - launches0
    import ctypes
    kms = (ctypes.c_double * 8)()
    nk, ne = ctypes.c_int(0), ctypes.c_int(0)
    _lib.check(lib.ccm_profile_end(ev.handle, kms, 8, ctypes.byref(nk), ctypes.byref(ne)))
    names = ["tc_prep", "tc_forward", "tc_backward", "tc_finalize"]
    kernels = {names[i]: kms[i] / max(ne.value, 1) for i in range(min(nk.value, 4))}
    elapsed_ms = max_over_ranks(world, elapsed_ms)
    value = world * args.steps / (elapsed_ms / 1e3)
    res = ev.result()
    f_gpu = res.fx
    g_gpu = gd.cpu().numpy()

    # end to end through the host-pointer ABI (pinned host buffers)
    xh = torch.from_numpy(x.copy()).pin_memory()
    gh = torch.empty_like(xh).pin_memory()
    fx = ctypes.c_double(0.0)
    xp = ctypes.cast(xh.data_ptr(), ctypes.POINTER(ctypes.c_float))
    gp = ctypes.cast(gh.data_ptr(), ctypes.POINTER(ctypes.c_float))
    for _ in range(2):
        _lib.check(lib.ccm_evaluate_host(ev.handle, xp, gp, xh.numel(), ctypes.byref(fx)))
    barrier(world)
    e_start, e_end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e_start.record(stream)
    for _ in range(args.e2e_steps):
        _lib.check(lib.ccm_evaluate_host(ev.handle, xp, gp, xh.numel(), ctypes.byref(fx)))
    e_end.record(stream)
    e_end.synchronize()
    e2e_ms = max_over_ranks(world, e_start.elapsed_time(e_end))
    e2e_value = world * args.e2e_steps / (e2e_ms / 1e3)
    # the bytes each call copied (the padding states of x and g stay on their side
    # when x's are zero, as they are here)
    h2d_b, d2h_b = ctypes.c_longlong(0), ctypes.c_longlong(0)
    _lib.check(lib.ccm_host_copy_bytes(ev.handle, ctypes.byref(h2d_b), ctypes.byref(d2h_b)))
    ev.close()

    out = None
    if rank == 0:
        peaks, peak_kind = measured_peaks()
        peak_burst = float(peaks.get("bf16_tflops", peaks.get("bf16_tflops_sustained")))
        peak_sustained = float(peaks.get("bf16_tflops_sustained", peak_burst))
        peak, peak_name, peak_why = tensor_peak(peaks, peak_kind, clocks, elapsed_ms)

        flops = 2.0 * N * (21 * L) ** 2
        dom = max(("tc_forward", "tc_backward"), key=lambda k: kernels.get(k, 0.0))
        dom_ms = kernels.get(dom, float("nan"))
        achieved = flops / (dom_ms / 1e3) / 1e12
        traffic = traffic_from_profiles(dom, args.path)
        # tensor-core flops actually issued by the dominant kernel: every split term,
        # the padded shapes (S = 256 slots per 12 columns, rows padded to 256) and,
        # for the backward, both products O^T R and R^T O on the upper-triangle tiles
        # bf16-equivalent products per element: 2 (hi+lo), 3 (three terms); the integer
        # path does three 8-bit products at twice the bf16 rate = 1.5
        nsplit = {"tc_bf16x3": 3, "tc_i8x3": 1.5, "tc_i8sp": 1.5}.get(args.path, 2)
        Npad = (N + 255) // 256 * 256
        if args.path == "tc_i8sp":
            # forward: 192-slot groups (9 columns) as N, K = 21 L padded to 256, three
            # 8-bit products at the 2:4-sparse rate (four times bf16): 0.75 per element;
            # backward: the 192-slot groups padded to 256-slot tiles
            SW = 192 * ((L + 8) // 9)
            KP = (21 * L + 255) // 256 * 256
            TB = (SW + 255) // 256
            executed = {"tc_forward": 2.0 * Npad * SW * KP * 0.75,
                        "tc_backward": TB * (TB + 1) / 2 * 256 * 256 * 2.0 * Npad * 2 * nsplit}[dom]
        else:
            T = (L + 11) // 12
            S = 256 * T
            executed = {"tc_forward": 2.0 * Npad * S * S * nsplit,
                        "tc_backward": T * (T + 1) / 2 * 256 * 256 * 2.0 * Npad * 2 * nsplit}[dom]
        executed_tf = executed / (dom_ms / 1e3) / 1e12

        # the dense integer and split-bf16 tensor-core paths on the same inputs, same
        # timing method
        others = {}
        for cpath in ("tc_i8x3", "tc_bf16x2"):
            if args.compare_steps <= 0 or world != 1 or cpath == args.path:
                continue
            be = cb.Evaluator(msa, weights=w, path=cpath, device=local)
            gb = torch.empty_like(xd)
            for _ in range(3):
                be.evaluate(xd, gb)
            torch.cuda.synchronize()
            bs = torch.cuda.ExternalStream(be.stream)
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(bs)
            for _ in range(args.compare_steps):
                _lib.check(lib.ccm_evaluate_async(be.handle, xd.data_ptr(), gb.data_ptr(), xd.numel()))
            b.record(bs)
            b.synchronize()
            bv = args.compare_steps / (a.elapsed_time(b) / 1e3)
            be.evaluate(xd, gb)
            f_b = be.result().fx
            g_b = gb.cpu().numpy()
            be.close()
            others[cpath] = {"evals_per_s": bv, "steps": args.compare_steps,
                             "arithmetic": PATH_ARITHMETIC[cpath],
                             "precision": None if args.no_precision
                             else precision_block(msa, w, x, g_b, f_b, L)}

        plain = None
        if args.plain_steps > 0 and world == 1:
            pe = cb.Evaluator(msa, weights=w, path="simt_f32", device=local)
            g2 = torch.empty_like(xd)
            pe.evaluate(xd, g2)
            torch.cuda.synchronize()
            ps = torch.cuda.ExternalStream(pe.stream)
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(ps)
            for _ in range(args.plain_steps):
                _lib.check(lib.ccm_evaluate_async(pe.handle, xd.data_ptr(), g2.data_ptr(), xd.numel()))
            b.record(ps)
            b.synchronize()
            pv = args.plain_steps / (a.elapsed_time(b) / 1e3)
            f_plain = pe.result().fx
            g_plain = g2.cpu().numpy()
            pe.close()
            plain = {"evals_per_s": pv, "tc_over_plain": value / pv,
                     "path": "plain FP32 CUDA-core kernels (ccm_simt.cu)"}
        prec = None
        if not args.no_precision:
            prec = {args.path: precision_block(msa, w, x, g_gpu, f_gpu, L)}
            if plain is not None:
                prec["simt_f32"] = precision_block(msa, w, x, g_plain, f_plain, L)
        ref_cuda = None
        if args.ref_cuda_steps > 0 and world == 1:
            ref_cuda = reference_cuda_timing(msa, x, xd, args.ref_cuda_steps,
                                             not args.no_precision)
        cpu = None
        if not args.no_cpu_baseline and world == 1:
            v, n_ev, kind, cores = cpu_reference_timing(msa, x, args.cpu_budget_s, 10)
            cpu = {"value": v, "unit": UNIT, "cores": cores, "kind": kind,
                   "sample": f"{n_ev} full evaluation(s) of the L=300 N=5000 workload "
                             f"(median), evaluate_cpu_omp with all {cores} host threads"}
            if kind == "reference":
                # the serial evaluate_cpu beside it (one evaluation, about 10 s)
                v1, n1, _, _ = cpu_reference_timing(msa, x, 0.0, 1, omp=False)
                cpu["serial_evaluate_cpu"] = {"value": v1, "unit": UNIT, "cores": 1,
                                              "sample": f"{n1} full evaluation, evaluate_cpu"}
        out = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": elapsed_ms / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": PATH_DTYPE[args.path],
            "data": "synthetic",
            "config": workload_config(cfg, world),
            "impl_detail": {"path": args.path, "arithmetic": PATH_ARITHMETIC[args.path]},
            "roofline": {"bound": "tensor", "kernel": dom, "achieved": achieved, "peak": peak,
                         "unit": "TFLOP/s", "frac": achieved / peak,
                         "peak_source": f"{peak_kind} {peak_name} ({peak_why})",
                         "frac_vs_burst": achieved / peak_burst,
                         "frac_vs_sustained": achieved / peak_sustained,
                         "flops_per_launch": flops, "traffic": traffic,
                         "executed_flops_per_launch": executed,
                         "executed_tflops": executed_tf, "executed_frac": executed_tf / peak,
                         "executed_note": "executed_frac compares 8-bit (integer) MMA work, "
                                          "counted in bf16-equivalent FLOPs, with the bf16 peak"
                                          if args.path in ("tc_i8x3", "tc_i8sp") else None},
            "kernels_ms_per_launch": kernels,
            "cpu_baseline": cpu,
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": h2d_b.value,
                    "d2h_bytes_per_step": d2h_b.value,
                    "api": "ccm_evaluate_host (pinned host x and g)"},
            "gpu_launches": int(launches),
            "clocks": clocks,
            "plain_f32": plain,
            "tc_i8x3": others.get("tc_i8x3"),
            "tc_bf16x2": others.get("tc_bf16x2"),
            "reference_cuda": ref_cuda,
            "precision": prec,
            "init_ms": {"weights": init_ms},
        }
        if world == 1 and not args.no_extras:
            # the other two workloads of the same library, after the headline's timed
            # region (which they do not touch): the ragged batch to convergence and
            # the large alignment's device-side solve, each as its own line would
            # report it (the large solve without its ~40 s CPU sample)
            for key, fn in (("batch256", lambda: run_batch(args, world, rank, local, False)),
                            ("L1000_N20000",
                             lambda: run_large(args, world, rank, local, False, False))):
                try:
                    out[key] = fn()
                except Exception as exc:  # the headline line is printed regardless
                    out[key] = {"error": f"{type(exc).__name__}: {exc}"}
        emit((out))
    barrier(world)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
