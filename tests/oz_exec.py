"""numpy executor of the split-precision H*psi tables (test helper, CPU only).

It repeats the device arithmetic step by step -- row maxima, power-of-two
scales, truncated radix-128 digits in the tile-ready layout, exact integer
slice products per diagonal over each family's concatenated k-blocks, the
FP64 epilogue in the kernel's order, the products' pi maxima -- and checks
the table indices on the way (every split inside its pool, every output tile
covered once per launch), so that the split-precision plan can be verified
without a GPU.
"""
import math

import numpy as np

from tests.plan_exec import merged_ops


def _pow2_of(m):
    """2^(E+1) for m = 1.f * 2^E (the device reads it off the exponent bits); 0 for m = 0."""
    m = np.asarray(m, dtype=np.float64)
    out = np.zeros_like(m)
    nz = m > 0
    out[nz] = np.ldexp(1.0, np.maximum(np.frexp(m[nz])[1], -1022))
    return out


class _Machine:
    def __init__(self, plan, oz, psi):
        ex, oe = plan["ex"], oz["ex"]
        self.plan, self.oz, self.ex, self.oe = plan, oz, ex, oe
        self.S, self.BN = oe.slices, oe.tile_n
        self.ops = merged_ops(plan)
        self.psi = np.concatenate([psi, np.zeros(8)])
        self.scr = np.full(ex.scratch_len + 8, np.nan)
        self.out = np.full(max(ex.psi_len, 1), np.nan)
        self.pack = np.zeros(oe.sta_pack + oe.dyn_pack, dtype=np.int8)
        self.scales = np.zeros(oe.n_scales)
        self.spaces = {1: self.ops, 2: self.psi, 3: self.scr}

    def _matrix(self, j):
        base = self.spaces[j.space]
        r = np.arange(j.nrows, dtype=np.int64)[:, None]
        k = np.arange(j.K, dtype=np.int64)[None, :]
        return j.coef * base[j.src_off + r * j.rs + k * j.ks]

    def run_max(self, jobs, n):
        for i in range(n):
            j = jobs[i]
            if not j.want_max:
                continue
            A = np.abs(self._matrix(j))
            m = np.max(A, axis=1)
            idx = j.scale_idx + np.arange(j.nrows)
            self.scales[idx] = np.maximum(self.scales[idx], m)
            if j.want_max == 2:
                # a psi cell split both ways: its column maxima too, from dst
                cidx = j.dst + np.arange(j.K)
                self.scales[cidx] = np.maximum(self.scales[cidx], np.max(A, axis=0))

    def run_split(self, jobs, n):
        S = self.S
        for i in range(n):
            j = jobs[i]
            if not j.want_split:
                continue
            nkb = -(-j.K // 32)
            rows = j.gtot * 8
            X = np.zeros((rows, nkb * 32))
            X[:j.nrows, :j.K] = self._matrix(j)
            sc = np.zeros(rows)
            sc[:j.nrows] = _pow2_of(self.scales[j.scale_idx:j.scale_idx + j.nrows])
            with np.errstate(divide="ignore", invalid="ignore"):
                t = np.where(sc[:, None] > 0, X * np.where(sc > 0, 1.0 / np.where(sc > 0, sc, 1.0), 0.0)[:, None], 0.0)
            dig = np.zeros((S, rows, nkb * 32), dtype=np.int64)
            for q in range(S):
                t = t * 128.0
                a = np.trunc(t)
                t = t - a
                dig[q] = a.astype(np.int64)
            assert np.all(np.abs(dig) <= 127)
            # split row sr -> tile, group; [tile][kb][p][g][c][r8][16]
            for jr in range(0, rows, 8):
                sr = j.row0 + jr
                tt, rl = divmod(sr, j.R)
                gt = j.R // 8 if tt < j.ntiles - 1 else j.gt_last
                g = rl // 8
                assert g < gt
                tile = j.dst + tt * j.nkb * S * (j.R // 8) * 256
                for kb in range(nkb):
                    for q in range(S):
                        o = tile + ((j.kb0 + kb) * S + q) * gt * 256 + g * 256
                        assert 0 <= o and o + 256 <= len(self.pack)
                        blk = dig[q, jr:jr + 8, kb * 32:(kb + 1) * 32].reshape(8, 2, 16).transpose(1, 0, 2)
                        self.pack[o:o + 256] = blk.reshape(-1).astype(np.int8)

    def tile_digits(self, base, nkb_tot, tile_groups, t, g, kb0, nkb):
        """Slices (S, 8*g, 32*nkb) of tile t (g groups; full tiles have tile_groups) of a split."""
        S = self.S
        out = np.zeros((S, g * 8, nkb * 32), dtype=np.int64)
        tb = base + t * nkb_tot * S * tile_groups * 256
        for kb in range(nkb):
            o = tb + (kb0 + kb) * S * g * 256
            assert 0 <= o and o + S * g * 256 <= len(self.pack)
            b = self.pack[o:o + S * g * 256].astype(np.int64).reshape(S, g, 2, 8, 16)
            out[:, :, kb * 32:(kb + 1) * 32] = b.transpose(0, 1, 3, 2, 4).reshape(S, g * 8, 32)
        return out

    def accum(self, A, B):
        """sum_d 128^-(d+2) D_d, D_d = sum_{p+q=d+2} A_p B_q^T, summed from the last diagonal down."""
        S = self.S
        D = [0] * S
        for pa in range(1, S + 1):
            for qb in range(1, S + 2 - pa):
                D[pa + qb - 2] = D[pa + qb - 2] + A[pa - 1] @ B[qb - 1].T
        acc = np.zeros((A.shape[1], B.shape[1]))
        for d in range(S - 1, -1, -1):
            if not isinstance(D[d], int):
                assert np.max(np.abs(D[d])) < 2 ** 31
                acc = acc + D[d].astype(np.float64) * (2.0 ** (-7 * (d + 2)))
        return acc

    def run_items(self, items, n, covered):
        oz = self.oz
        for ii in range(n):
            it = items[ii]
            assert it.M in (64, 128) and it.mrows <= it.M and it.N % 16 == 0 and it.ncols <= it.N <= self.BN
            assert it.fam_end - it.fam_begin <= 3
            ta, tb = it.row0 // 128, it.col0 // self.BN
            ga, gb = -(-it.mrows // 8), it.N // 8

            def operands(sg):
                A = self.tile_digits(sg.a_base, sg.a_nkb, 16, ta, ga, sg.a_kb0, sg.nkb)
                B = self.tile_digits(sg.b_base, sg.b_nkb, self.BN // 8, tb, gb, sg.b_kb0, sg.nkb)
                return A, B

            c = oz["cells"][it.cell]
            key = (it.cell, it.row0, it.col0)
            assert key not in covered
            covered.add(key)
            rows = it.row0 + np.arange(it.mrows)
            cols = it.col0 + np.arange(it.ncols)
            idx = c.off + rows[:, None] + cols[None, :] * c.ld
            tot = np.zeros((it.mrows, it.ncols))
            for f in range(it.fam_begin, it.fam_end):
                fm = oz["fams"][f]
                As, Bs = zip(*[operands(oz["segs"][sgi]) for sgi in range(fm.seg_begin, fm.seg_end)])
                A = np.concatenate(As, axis=2)[:, :it.mrows]
                B = np.concatenate(Bs, axis=2)[:, :it.ncols]
                # the device accumulates at most kb_piece k-blocks in int32, then adds the pieces
                kp = 32 * ((2 ** 31 - 1) // (32 * self.S * 127 * 127))
                acc = sum(self.accum(A[:, :, k0:k0 + kp], B[:, :, k0:k0 + kp]) for k0 in range(0, A.shape[2], kp))
                rs = _pow2_of(self.scales[fm.rs_idx + rows])
                cs = _pow2_of(self.scales[fm.cs_idx + cols])
                tot = tot + (acc * rs[:, None]) * cs[None, :]
            if it.kind == 0:
                if it.init:
                    old = np.zeros((it.mrows, it.ncols))
                    tasks = self.plan["tasks2"]
                    for a in range(c.a_begin, c.a_end):
                        t = tasks[a]
                        b = self.spaces[t.L.space]
                        old = old + t.coef * b[t.L.off + cols[None, :] * t.L.ld + rows[:, None]]
                else:
                    old = self.out[idx]
                self.out[idx] = old + tot
            else:
                # a tile of a product stack: each row stored to the product it
                # belongs to, and that row's pi raised by its maximum; the
                # stack's padding rows (products start on 8-row groups) are zero
                assert it.fam_end - it.fam_begin == 1 and not it.init
                prods = [oz["prod_rows"][k] for k in range(c.a_begin, c.a_end)]
                for i, R in enumerate(rows):
                    hit = [q for q in prods if q.row_begin <= R < q.row_begin + q.rows]
                    if not hit:
                        assert np.all(tot[i] == 0.0)
                        continue
                    q = hit[0]
                    rr = int(R - q.row_begin)
                    self.scr[q.off + rr + cols * q.ld] = tot[i]
                    self.scales[q.pi + rr] = max(self.scales[q.pi + rr], float(np.max(np.abs(tot[i]))))


def execute_ozaki(plan, oz, psi):
    """H*psi through the split-precision tables, as the device runs them."""
    m = _Machine(plan, oz, psi)
    oe = m.oe
    # once per step
    m.run_max(oz["sta_mjobs"], oe.n_sta_mjobs)
    m.run_split(oz["sta_jobs"], oe.n_sta_jobs)
    # per H*psi
    m.scales[oe.rho0:] = 0.0
    m.run_max(oz["psi_mjobs"], oe.n_psi_mjobs)
    m.run_split(oz["psi_jobs"], oe.n_psi_jobs)
    for n_items, cta, n_cta in ((oe.n_items1, oz["cta1"], oe.n_cta1), (oe.n_items2, oz["cta2"], oe.n_cta2)):
        b = [cta[i] for i in range(n_cta)]
        assert b[0] == 0 and b[-1] == n_items and all(x <= y for x, y in zip(b, b[1:])) and len(b) <= 149
    cov1 = set()
    m.run_items(oz["items1"], oe.n_items1, cov1)
    m.run_max(oz["prod_mjobs"], oe.n_prod_mjobs)
    m.run_split(oz["prod_jobs"], oe.n_prod_jobs)
    cov2 = set()
    m.run_items(oz["items2"], oe.n_items2, cov2)
    # every phase-1 product was written where it is read
    ex = plan["ex"]
    for ci in range(ex.n_cells1):
        c = plan["cells1"][ci]
        idx = c.off + np.arange(c.N)[:, None] * c.ld + np.arange(c.M)[None, :]
        assert np.all(np.isfinite(m.scr[idx])), "product %d not fully written" % ci
    return m.out[:ex.psi_len]
