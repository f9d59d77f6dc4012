"""numpy executor of the split-precision H*psi tables (test helper, CPU only).

It repeats the device arithmetic step by step -- row scales, truncated int8
slices, exact integer slice products per diagonal, the FP64 epilogue in the
kernel's order, the per-cell sums -- and checks every table index on the way
(pack offsets inside their pools, each product and slot entry written exactly
once), so that the split-precision plan can be verified without a GPU.
"""
import math

import numpy as np

from tests.plan_exec import merged_ops


def _rows(base, sp, nrows, K):
    """Matrix (nrows x K) of a split: element (r, k) = base[src_off + r*rs + k*ks]."""
    r = np.arange(nrows, dtype=np.int64)[:, None]
    k = np.arange(K, dtype=np.int64)[None, :]
    return base[sp.src_off + r * sp.rs + k * sp.ks]


def _split(base, sp, s, pack, sig):
    """oz_split_kernel: per-row power-of-two scale and s truncated radix-128 digits."""
    X = _rows(base, sp, sp.nrows, sp.K)
    out = np.zeros((s, sp.nrows, sp.K_pad), dtype=np.int64)
    for r in range(sp.nrows):
        mx = float(np.max(np.abs(X[r]))) if sp.K else 0.0
        if mx > 0.0:
            e = math.frexp(mx)[1]
            sig[sp.sig_off + r] = math.ldexp(1.0, e)
            t = np.ldexp(X[r], -e)
            for q in range(s):
                t = t * 128.0
                a = np.trunc(t)
                t = t - a
                out[q, r, :sp.K] = a.astype(np.int64)
        else:
            sig[sp.sig_off + r] = 0.0
    assert np.all(np.abs(out) <= 127)
    end = sp.pack_off + s * sp.nrows * sp.K_pad
    assert 0 <= sp.pack_off and end <= len(pack)
    pack[sp.pack_off:end] = out.reshape(-1)


def _gemm(groups, ngroups, rows, items, nitems, s, bn, dyn_pack, dyn_sig, sta_pack, sta_sig, dst, written):
    # every (group, row tile, n tile) exactly once
    seen = set()
    for i in range(nitems):
        it = items[i]
        key = (it.group, it.row0, it.n0)
        assert key not in seen
        seen.add(key)
    expect = set()
    for gi in range(ngroups):
        g = groups[gi]
        for r0 in range(0, g.row_end - g.row_begin, 128):
            for n0 in range(0, g.N, bn):
                expect.add((gi, r0, n0))
    assert seen == expect
    w = 2.0 ** (-7 * np.arange(2, s + 2))
    for gi in range(ngroups):
        g = groups[gi]
        B = sta_pack[g.s_pack_off:g.s_pack_off + s * g.N * g.K_pad].reshape(s, g.N, g.K_pad)
        tau = sta_sig[g.tau_off:g.tau_off + g.N]
        nr = g.row_end - g.row_begin
        A = np.zeros((s, nr, g.K_pad), dtype=np.int64)
        for j in range(nr):
            R = rows[g.row_begin + j]
            for p in range(s):
                o = R.pack_off + p * R.slice_stride
                assert 0 <= o and o + g.K_pad <= len(dyn_pack)
                A[p, j] = dyn_pack[o:o + g.K_pad]
        diag = np.zeros((s, nr, g.N), dtype=np.int64)
        for p in range(1, s + 1):
            for q in range(1, s + 2 - p):
                diag[p + q - 2] += A[p - 1] @ B[q - 1].T
        assert np.max(np.abs(diag)) < 2 ** 31
        acc = np.zeros((nr, g.N))
        for d in range(s - 1, -1, -1):
            acc = acc + diag[d].astype(np.float64) * w[d]
        for j in range(nr):
            R = rows[g.row_begin + j]
            vals = acc[j] * (R.coef * dyn_sig[R.sig_idx]) * tau
            idx = R.dst_off + np.arange(g.N, dtype=np.int64) * R.dst_stride
            space = dst[R.dst_space]
            assert idx.min() >= 0 and idx.max() < len(space)
            space[idx] = vals
            written[R.dst_space][idx] += 1


def execute_ozaki(plan, oz, psi):
    """H*psi through the split-precision tables; returns (out, checks dict)."""
    ex, oe = plan["ex"], oz["ex"]
    s, bn = oe.slices, oe.tile_n
    ops = merged_ops(plan)
    psi = np.concatenate([psi, np.zeros(8)])
    scr = np.full(ex.scratch_len + 8, np.nan)
    slots = np.full(max(oe.slots_len, 1), np.nan)
    sta_pack = np.zeros(oe.sta_pack, dtype=np.int64)
    sta_sig = np.full(oe.sta_sig, np.nan)
    dyn_pack = np.zeros(oe.dyn_pack, dtype=np.int64)
    dyn_sig = np.full(oe.dyn_sig, np.nan)
    for i in range(oe.n_sta):
        assert oz["sta"][i].space == 1
        _split(ops, oz["sta"][i], s, sta_pack, sta_sig)
    for i in range(oe.n_dyn_a):
        assert oz["dyn_a"][i].space == 2
        _split(psi, oz["dyn_a"][i], s, dyn_pack, dyn_sig)
    written = {0: np.zeros(len(scr), dtype=np.int64), 1: np.zeros(len(slots), dtype=np.int64)}
    dst = {0: scr, 1: slots}
    _gemm(oz["groups_a"], oe.n_groups_a, oz["rows_a"], oz["items_a"], oe.n_items_a, s, bn, dyn_pack, dyn_sig,
          sta_pack, sta_sig, dst, written)
    for i in range(oe.n_dyn_b):
        assert oz["dyn_b"][i].space == 3
        _split(scr, oz["dyn_b"][i], s, dyn_pack, dyn_sig)
    _gemm(oz["groups_b"], oe.n_groups_b, oz["rows_b"], oz["items_b"], oe.n_items_b, s, bn, dyn_pack, dyn_sig,
          sta_pack, sta_sig, dst, written)
    # cell sums
    out = np.full(max(ex.psi_len, 1), np.nan)
    spaces = {1: ops, 2: psi, 3: scr}
    tasks = plan["tasks2"]
    for ci in range(oe.n_sums):
        c = oz["sums"][ci]
        v = np.zeros((c.N, c.M))
        for j in range(c.s_begin, c.s_end):
            o = oz["slot_offs"][j]
            v = v + slots[o:o + c.M * c.N].reshape(c.N, c.M)
        for a in range(c.a_begin, c.a_end):
            t = tasks[a]
            b = spaces[t.L.space]
            idx = t.L.off + np.arange(c.N)[:, None] * t.L.ld + np.arange(c.M)[None, :]
            v = v + t.coef * b[idx]
        idx = c.out_off + np.arange(c.N)[:, None] * c.ld + np.arange(c.M)[None, :]
        out[idx] = v
    # phase-1 products and task slots: written exactly once where read
    cells1 = plan["cells1"]
    for ci in range(ex.n_cells1):
        c = cells1[ci]
        idx = c.off + np.arange(c.N)[:, None] * c.ld + np.arange(c.M)[None, :]
        assert np.all(written[0][idx] == 1)
    used = np.zeros(len(slots), dtype=bool)
    for ci in range(oe.n_sums):
        c = oz["sums"][ci]
        for j in range(c.s_begin, c.s_end):
            o = oz["slot_offs"][j]
            used[o:o + c.M * c.N] = True
    assert np.all(written[1][used] == 1)
    return out[:ex.psi_len]
