"""Synthetic batched block-GEMM workload of the grouped-GEMM benchmark.

The batched block-GEMM pattern of one two-site H*psi without its physics:
n_cells (N, S) sector pairs, each an output cell whose dimensions are drawn
log-uniform in [dmin, dmax]; each cell receives 4..16 Hamiltonian terms, a
term being one block GEMM coef * op(L) op(R) with op(L) M x K and op(R)
K x N.  K is the dimension of the operator sub-block the term touches: the
operators are block-sparse with 3x3 .. 12x12 sub-blocks, whose dimensions
are drawn log-uniform in [dmin, dmax] as well.  Entries are N(0, 1) FP64
(every operand is a window of one pool), recoupling weights coef are
U[-1, 1], and L / R are stored transposed with probability 1/2 (the
transposed environment operators of H*psi).  Seeded with numpy's MT19937.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field

import numpy as np

from .structs import TjGgCell, TjGgTerm


@dataclass
class GgBatch:
    cells: object            # ctypes array of TjGgCell
    terms: object            # ctypes array of TjGgTerm
    pool: np.ndarray
    out_len: int
    flops: float
    spec: dict = field(default_factory=dict)


def _logu(rng, lo, hi, n=None):
    return np.rint(np.exp(rng.uniform(np.log(lo), np.log(hi), n))).astype(np.int64)


def make_batch(n_cells: int = 400, dmin: int = 8, dmax: int = 1024, tmin: int = 4, tmax: int = 16,
               seed: int = 2024, pool_len: int = 1 << 24) -> GgBatch:
    rng = np.random.Generator(np.random.MT19937(seed))
    pool = rng.standard_normal(pool_len)
    cells = (TjGgCell * n_cells)()
    terms_py = []
    off = 0
    flops = 0.0
    nblk = []
    for c in range(n_cells):
        M, N = (int(x) for x in _logu(rng, dmin, dmax, 2))
        nt = int(rng.integers(tmin, tmax + 1))
        b = int(rng.integers(3, 13))          # sub-block grid of the term's operators
        kdims = _logu(rng, dmin, dmax, b)     # their sub-block dimensions
        nblk.append(b)
        t0 = len(terms_py)
        for _ in range(nt):
            K = int(kdims[rng.integers(0, b)])
            lt, rt = int(rng.integers(0, 2)), int(rng.integers(0, 2))
            lrows, lcols = (K, M) if lt else (M, K)
            rrows, rcols = (N, K) if rt else (K, N)
            lo = int(rng.integers(0, pool_len - lrows * lcols + 1))
            ro = int(rng.integers(0, pool_len - rrows * rcols + 1))
            terms_py.append((lo, ro, lrows, rrows, K, lt, rt, float(rng.uniform(-1.0, 1.0))))
            flops += 2.0 * M * N * K
        cells[c] = TjGgCell(off, M, N, t0, len(terms_py))
        off += M * N
    terms = (TjGgTerm * len(terms_py))()
    for i, (lo, ro, lld, rld, K, lt, rt, coef) in enumerate(terms_py):
        terms[i] = TjGgTerm(lo, ro, lld, rld, K, lt, rt, 0, coef)
    spec = {"cells": n_cells, "terms": len(terms_py), "dims": [dmin, dmax], "terms_per_cell": [tmin, tmax],
            "operator_subblocks": [3, 12], "seed": seed, "generator": "numpy MT19937",
            "pool_doubles": pool_len}
    return GgBatch(cells, terms, pool, off, flops, spec)


def _window(pool, off, ld, rows, cols):
    return pool[off:off + ld * cols].reshape(cols, ld).T[:rows, :]


def reference(batch: GgBatch, which=None) -> dict:
    """numpy result of the cells in `which` (all by default): {cell: M x N array}."""
    res = {}
    idx = range(len(batch.cells)) if which is None else which
    for c in idx:
        cl = batch.cells[c]
        y = np.zeros((cl.M, cl.N))
        for t in range(cl.t_begin, cl.t_end):
            x = batch.terms[t]
            L = _window(batch.pool, x.l_off, x.l_ld, *((x.K, cl.M) if x.l_trans else (cl.M, x.K)))
            R = _window(batch.pool, x.r_off, x.r_ld, *((cl.N, x.K) if x.r_trans else (x.K, cl.N)))
            y += x.coef * ((L.T if x.l_trans else L) @ (R.T if x.r_trans else R))
        res[c] = y
    return res


def cell_view(batch: GgBatch, out: np.ndarray, c: int) -> np.ndarray:
    cl = batch.cells[c]
    return out[cl.out_off:cl.out_off + cl.M * cl.N].reshape(cl.N, cl.M).T
