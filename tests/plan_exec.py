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


def execute(plan, psi: np.ndarray) -> np.ndarray:
    ex = plan["ex"]
    ops = plan["ops"].copy()
    for r in range(ex.n_merges):
        m = plan["merges"][r]
        acc = np.zeros(m.n)
        for j in range(m.s_begin, m.s_end):
            s = plan["merge_src"][j]
            acc = acc + plan["merge_coef"][j] * ops[s:s + m.n]
        ops[m.dst:m.dst + m.n] = acc
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
