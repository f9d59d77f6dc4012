"""Correlation functions of a DMRG wavefunction over the library's entry points.

The reference measures after its last half-sweep (Measurement, code/tjsq/
main.f90:191-332): one-site operators are placed at a site of the system or
environment chain and carried to the current blocks through the stored
bases and truncations (Get_*_oper_*, Change_*_oper_*, get_sys.f90:764-1238);
two operators of the same block are multiplied with the 3j recoupling first
(Get_sys2b, measure.f90:2785-2819, with block_mul_block_ndia); the
contractions with the wavefunction are the nine kernels of measure.f90.
This module restates the driver Get_density_cor (measure.f90:3110-3223) that
gives <O1_i O2_j> for a reference site i and the sites j of its row -- the
spin correlation <S_i . S_j> (st_sd, st_sd), the density correlation
<n_i n_j> (num_elec, num_elec) and the single-particle correlation
(st_elec_up, st_elec_down) -- without its file output.

A backend provides get_oper, change_oper, update_trun, block_mul_block_ndia
and correlator (`DeviceBackend` in grand_sql_tj_b200.lib runs them on the
B200 through the C ABI).
"""
from __future__ import annotations

import math
from typing import Dict, Tuple

from .structs import PackedChain, block_transfer_trans


class Chains:
    """The measurement tables of both sides (sys_bsm / systruns and env_bsm /
    envtruns of the reference), from a sweep driver's stored bases and
    truncations, for the wavefunction `wave`."""

    def __init__(self, dmrg, wave, trun_idx: int = 1):
        self.sys_len, self.env_len = wave.sys_len, wave.env_len
        self.trun_idx = trun_idx
        self.sys_bases = {i: dmrg.sysbs[i] for i in range(2, self.sys_len + 1) if i in dmrg.sysbs}
        self.env_bases = {i: dmrg.envbs[i] for i in range(2, self.env_len + 1) if i in dmrg.envbs}
        self.sys_truns = {i: dmrg.systruns[i] for i in range(2, self.sys_len + 1) if i in dmrg.systruns}
        self.env_truns = {i: dmrg.envtruns[i] for i in range(2, self.env_len + 1) if i in dmrg.envtruns}
        self.sys = PackedChain(self.sys_len, self.sys_bases, self.sys_truns, trun_idx)
        self.env = PackedChain(self.env_len, self.env_bases, self.env_truns, trun_idx)


def get_sys2b(be, ch: Chains, idx1: int, idx2: int, oper1, oper2, flag: str):
    """Get_sys2b (measure.f90:2785-2819): O1 at idx1 times O2 at idx2 (idx1 <
    idx2 <= sys_len - 1), coupled to a scalar and carried to the system block."""
    n1 = be.get_oper(0, 0, ch.sys, oper1, idx1, idx2, False, flag)
    n2 = be.get_oper(0, 0, ch.sys, oper2, idx2, idx2, False, flag)
    new = be.block_mul_block_ndia(n1, "N", n2, "N", 1.0, 0, ch.sys_bases[idx2])
    if idx2 > ch.trun_idx:
        new = be.update_trun(1, new, ch.sys_truns[idx2])
    return be.change_oper(0, 1, ch.sys, new, idx2, ch.sys_len - 1, True, flag)


def density_cor(be, ch: Chains, wave, oper1, oper2, flag: str, sid1: int, ny: int, num_site: int,
                ij: int = 0) -> Dict[Tuple[int, int], float]:
    """Get_density_cor(oper_ndia, oper1, oper2, wave, trun_idx, Flags, ..., xi = xj = sid1, ij)
    (measure.f90:3110-3223): <oper1_sid1 oper2_j> for the sites j = sid1 + ny + ij,
    sid1 + 2 ny + ij, ... of the system block and every later site j of
    sid1's row, scaled as the reference scales it (sqrt(1 + d), and -1 for d = 2)."""
    sys_len, env_len = ch.sys_len, ch.env_len
    sys_bs, env_bs = ch.sys_bases[sys_len], ch.env_bases[env_len]
    d = oper1.down_dif
    scale = math.sqrt(1.0 + d) * (-1.0 if d == 2 else 1.0)
    out = {}
    for sid2 in range(sid1 + ny + ij, sys_len, ny):
        op = get_sys2b(be, ch, min(sid1, sid2), max(sid1, sid2), oper1, oper2, flag)
        out[(sid1, sid2)] = be.correlator("measure_sys_block", op, None, sys_bs, None, wave) * scale
    n1 = be.get_oper(0, 0, ch.sys, oper1, sid1, sid1, sid1 > ch.trun_idx, flag)
    sys_oper = be.change_oper(0, 0, ch.sys, n1, sid1, sys_len - 1, True, flag)
    tr2 = block_transfer_trans(oper2) if oper2.down_dif == 1 else oper2
    for sid3 in range(sys_len, num_site + 1):
        if (sid1 + ij - sid3) % ny != 0:   # mod(sid1+ij-sid3, ny) >= 0 for sid3 > sid1: same row
            continue
        if sid3 == sys_len:
            value = be.correlator("sys_block_site_cor_ndia", sys_oper, tr2, sys_bs, None, wave, flag)
        elif sid3 == sys_len + 1:
            value = be.correlator("sys_block_env_site_cor_ndia", sys_oper, tr2, sys_bs, env_bs, wave, flag)
        else:
            eid1 = num_site - sid3 + 1
            n2 = be.get_oper(1, 0, ch.env, oper2, eid1, eid1, eid1 > ch.trun_idx, flag)
            env_oper = be.change_oper(1, 0, ch.env, n2, eid1, env_len - 1, True, flag)
            if oper2.down_dif != 0:
                env_oper = block_transfer_trans(env_oper)
            value = be.correlator("sys_block_env_block_cor_ndia", sys_oper, env_oper, sys_bs, env_bs, wave, flag)
        out[(sid1, sid3)] = value * scale
    return out
