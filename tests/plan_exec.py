"""numpy executor of an exported H*psi plan (test helper, CPU only).

It performs exactly the arithmetic the device kernels perform -- merged
operator sums, phase-1 products, phase-2 cell accumulation -- so that the
plan compiler can be checked against the oracle without a GPU.
"""
import numpy as np
from numpy.lib.stride_tricks import as_strided


def _view(base, op, rows, cols):
    a = base[op.off:]
    if op.trans == 0:
        return as_strided(a, shape=(rows, cols), strides=(8, 8 * op.ld))
    return as_strided(a, shape=(rows, cols), strides=(8 * op.ld, 8))


def merged_ops(plan) -> np.ndarray:
    """The operator space after the hmerge sums (what the device computes once per step)."""
    ex = plan["ex"]
    ops = plan["ops"].copy()
    for r in range(ex.n_merges):
        m = plan["merges"][r]
        acc = np.zeros(m.n)
        for j in range(m.s_begin, m.s_end):
            s = plan["merge_src"][j]
            acc = acc + plan["merge_coef"][j] * ops[s:s + m.n]
        ops[m.dst:m.dst + m.n] = acc
    return ops


def execute(plan, psi: np.ndarray) -> np.ndarray:
    ex = plan["ex"]
    ops = merged_ops(plan)
    scr = np.zeros(ex.scratch_len + 8)
    out = np.zeros(max(ex.psi_len, 1))
    psi = np.concatenate([psi, np.zeros(8)])
    spaces = {1: ops, 2: psi, 3: scr}

    def run(cells, tasks, ncell, dst):
        for ci in range(ncell):
            c = cells[ci]
            y = np.zeros((c.M, c.N))
            for ti in range(c.t_begin, c.t_end):
                t = tasks[ti]
                if t.R.space == 0:
                    y += t.coef * _view(spaces[t.L.space], t.L, c.M, c.N)
                else:
                    y += t.coef * (_view(spaces[t.L.space], t.L, c.M, t.K) @ _view(spaces[t.R.space], t.R, t.K, c.N))
            v = as_strided(dst[c.off:], shape=(c.M, c.N), strides=(8, 8 * c.ld))
            v[...] = y

    run(plan["cells1"], plan["tasks1"], ex.n_cells1, scr)
    run(plan["cells2"], plan["tasks2"], ex.n_cells2, out)
    return out[:ex.psi_len]


def execute_items(plan, psi: np.ndarray, tile: int = 64) -> np.ndarray:
    """Like execute(), but through the work items and reduce records, as the device does."""
    ex = plan["ex"]
    ops = merged_ops(plan)
    scr = np.zeros(ex.scratch_len + 8)
    out = np.full(max(ex.psi_len, 1), np.nan)
    psi = np.concatenate([psi, np.zeros(8)])
    spaces = {1: ops, 2: psi, 3: scr}

    def run(cells, tasks, items, nitem, reds, nred, dst):
        slots = {}
        for ii in range(nitem):
            it = items[ii]
            c = cells[it.cell]
            rows, cols = min(tile, c.M - it.row0), min(tile, c.N - it.col0)
            y = np.zeros((rows, cols))
            for ti in range(it.tb, it.te):
                t = tasks[ti]
                L = _view(spaces[t.L.space], t.L, c.M, t.K)[it.row0:it.row0 + rows]
                R = _view(spaces[t.R.space], t.R, t.K, c.N)[:, it.col0:it.col0 + cols]
                y += t.coef * (L @ R)
            for ti in range(it.ab, it.ae):
                t = tasks[ti]
                y += t.coef * _view(spaces[t.L.space], t.L, c.M, c.N)[it.row0:it.row0 + rows, it.col0:it.col0 + cols]
            if it.slot < 0:
                v = as_strided(dst[c.off:], shape=(c.M, c.N), strides=(8, 8 * c.ld))
                v[it.row0:it.row0 + rows, it.col0:it.col0 + cols] = y
            else:
                slots[it.slot] = y
        for ri in range(nred):
            rd = reds[ri]
            c = cells[rd.cell]
            rows, cols = min(tile, c.M - rd.row0), min(tile, c.N - rd.col0)
            y = np.zeros((rows, cols))
            for k in range(rd.nslot):
                y = y + slots[rd.slot0 + k]
            for ti in range(rd.ab, rd.ae):
                t = tasks[ti]
                y += t.coef * _view(spaces[t.L.space], t.L, c.M, c.N)[rd.row0:rd.row0 + rows, rd.col0:rd.col0 + cols]
            v = as_strided(dst[c.off:], shape=(c.M, c.N), strides=(8, 8 * c.ld))
            v[rd.row0:rd.row0 + rows, rd.col0:rd.col0 + cols] = y

    run(plan["cells1"], plan["tasks1"], plan["items1"], ex.n_items1, plan["red1"], ex.n_red1, scr)
    run(plan["cells2"], plan["tasks2"], plan["items2"], ex.n_items2, plan["red2"], ex.n_red2, out)
    return out[:ex.psi_len]
