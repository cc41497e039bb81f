"""Seeded synthetic multiple sequence alignments.

The reference ships a single real alignment (example/1atzA.aln, 75 columns)
and names no public benchmark set, so the workloads are synthetic MSAs over
the reference's 21-letter alphabet (20 amino acids + gap = 20,
src/sequence.c:10-27), generated as follows:

* per column j, amino-acid frequencies p_j ~ Dirichlet(0.5 * 1_20);
* each cell is a gap with probability ``gap_frac``, else drawn from p_j;
* ``n_pairs`` planted coupled column pairs on disjoint columns: for each pair
  (i, j) the two cells of every row are redrawn jointly from a random 21x21
  table with Dirichlet(0.5) weights over its 441 cells;
* optionally a fraction of rows are near-duplicates: a copy of a random
  earlier row with 5-25 % of its positions redrawn from the column model, so
  that pairwise identities straddle the 0.8 reweighting threshold.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

Q = 21


@dataclass(frozen=True)
class MSAConfig:
    name: str
    ncol: int
    nrow: int
    n_pairs: int = 0
    gap_frac: float = 0.1
    dup_frac: float = 0.0
    seed: int = 0


# Workloads (columns L, rows N, planted pairs, gaps, duplicates, seed).
SMALL_75x1000 = MSAConfig("L75_N1000", 75, 1000, n_pairs=30, seed=1)
PRECISION_300x5000 = MSAConfig("L300_N5000", 300, 5000, n_pairs=150, seed=2)
LARGE_1000x20000 = MSAConfig("L1000_N20000", 1000, 20000, n_pairs=0, gap_frac=0.2,
                             dup_frac=0.3, seed=3)
AUTOGRAD_150x2000 = MSAConfig("L150_N2000", 150, 2000, seed=5)


def generate(cfg: MSAConfig) -> np.ndarray:
    """uint8 (nrow, ncol) row-major MSA with states 0..20 (20 = gap)."""
    rng = np.random.Generator(np.random.PCG64(cfg.seed))
    L, N = cfg.ncol, cfg.nrow
    freqs = rng.dirichlet(np.full(Q - 1, 0.5), size=L)            # (L, 20)
    cdf = np.cumsum(freqs, axis=1)
    cdf[:, -1] = 1.0

    def draw_columns(rows: int, cols: np.ndarray) -> np.ndarray:
        u = rng.random((rows, cols.size))
        out = np.empty((rows, cols.size), dtype=np.uint8)
        for t, j in enumerate(cols):
            out[:, t] = np.searchsorted(cdf[j], u[:, t], side="right").clip(0, Q - 2)
        gap = rng.random((rows, cols.size)) < cfg.gap_frac
        out[gap] = Q - 1
        return out

    msa = draw_columns(N, np.arange(L))

    if cfg.n_pairs > 0:
        npairs = min(cfg.n_pairs, L // 2)
        cols = rng.permutation(L)[: 2 * npairs].reshape(npairs, 2)
        for (i, j) in cols:
            table = rng.dirichlet(np.full(Q * Q, 0.5))
            cell = rng.choice(Q * Q, size=N, p=table)
            msa[:, i] = (cell // Q).astype(np.uint8)
            msa[:, j] = (cell % Q).astype(np.uint8)

    if cfg.dup_frac > 0 and N > 1:
        ndup = int(round(cfg.dup_frac * N))
        rows = np.sort(rng.choice(np.arange(1, N), size=min(ndup, N - 1), replace=False))
        for r in rows:
            src = int(rng.integers(0, r))
            msa[r] = msa[src]
            frac = rng.uniform(0.05, 0.25)
            pos = np.nonzero(rng.random(L) < frac)[0]
            if pos.size:
                msa[r, pos] = draw_columns(1, pos)[0]
    return np.ascontiguousarray(msa)


def random_x(L: int, seed: int, v_sd: float = 0.1, w_sd: float = 0.01,
             symmetric: bool = True) -> np.ndarray:
    """Admissible parameters in the padded layout: V ~ N(0, v_sd^2), W ~ N(0, w_sd^2)
    tied symmetric W(b,k,a,j) = W(a,j,b,k), zero self blocks and zero padding."""
    rng = np.random.Generator(np.random.PCG64(seed))
    ns = L * (Q - 1)
    nsp = ns + 32 - ns % 32
    x = np.zeros(nsp + L * L * Q * 32, dtype=np.float32)
    x[:ns] = rng.normal(0.0, v_sd, ns).astype(np.float32)
    W = rng.normal(0.0, w_sd, (Q, L, Q, L)).astype(np.float32)     # [b,k,a,j]
    if symmetric:
        W = _symmetrise(W)
    idx = np.arange(L)
    W[:, idx, :, idx] = 0.0
    Wp = np.zeros((Q, L, 32, L), dtype=np.float32)
    Wp[:, :, :Q, :] = W
    x[nsp:] = Wp.reshape(-1)
    return x


def _symmetrise(W: np.ndarray) -> np.ndarray:
    """Mirror the strict upper triangle of W viewed as a (21L x 21L) matrix with
    rows (b,k) and columns (a,j), so that W(b,k,a,j) = W(a,j,b,k)."""
    n = W.shape[0] * W.shape[1]
    M = W.reshape(n, n)
    U = np.triu(M, 1)
    return (U + U.T + np.diag(np.diag(M))).reshape(W.shape).astype(np.float32)


def batch_workload(n: int = 256, seed0: int = 1000):
    """Ragged batch: n alignments, L ~ U[50, 400], N ~ logU[200, 20000], alignment i
    generated from seed seed0 + i (10 % gaps, L // 10 planted pairs)."""
    out = []
    for i in range(n):
        rng = np.random.Generator(np.random.PCG64(seed0 + i))
        L = int(rng.integers(50, 401))
        N = int(round(np.exp(rng.uniform(np.log(200), np.log(20000)))))
        out.append(generate(MSAConfig(f"batch{i}", L, N, n_pairs=L // 10, seed=seed0 + i)))
    return out
