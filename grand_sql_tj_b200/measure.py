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


def get_sys_two(be, ch: Chains, idx1: int, idx2: int, ops):
    """Get_sys_two (measure.f90:3798-3832): the singlet pair c+_idx1 c+_idx2
    (block_mul_block_ndia coupled to total spin 0) on the block of length idx2."""
    n1 = be.get_oper(0, 0, ch.sys, ops["elec_up"], idx1, idx2, False, "F")
    n2 = be.get_oper(0, 0, ch.sys, ops["elec_up"], idx2, idx2, False, "F")
    new = be.block_mul_block_ndia(n1, "N", n2, "N", 1.0, 0, ch.sys_bases[idx2])
    return be.update_trun(0, new, ch.sys_truns[idx2]) if idx2 > ch.trun_idx else new


def get_sys_two1(be, ch: Chains, idx2: int, idx3: int, idx4: int, pair, ops):
    """Get_sys_two1 (measure.f90:3835-3889): the pair operator of block length
    idx2 times c_idx3 (coupled to spin 1/2) times c_idx4 (coupled to spin 0),
    carried to the system block."""
    new = be.change_oper(0, 0, ch.sys, pair, idx2, idx3, False, "B")
    n1 = be.get_oper(0, 0, ch.sys, ops["elec_down"], idx3, idx3, False, "F")
    n2 = be.block_mul_block_ndia(new, "N", n1, "N", 1.0, 1, ch.sys_bases[idx3])
    n1 = be.update_trun(0, n2, ch.sys_truns[idx3]) if idx3 > ch.trun_idx else n2
    n12 = be.change_oper(0, 0, ch.sys, n1, idx3, idx4, False, "F")
    n2 = be.get_oper(0, 0, ch.sys, ops["elec_down"], idx4, idx4, False, "F")
    n3 = be.block_mul_block_ndia(n12, "N", n2, "N", 1.0, 0, ch.sys_bases[idx4])
    n1 = be.update_trun(1, n3, ch.sys_truns[idx4]) if idx4 > ch.trun_idx else n3
    return be.change_oper(0, 1, ch.sys, n1, idx4, ch.sys_len - 1, True, "B")


def get_scop_operator_env(be, ch: Chains, idx1: int, idx2: int, new_idx: int, truns: bool, ops):
    """Get_SCOP_Operator_Env (measure.f90:6211-6263), singlet 'S0': the pair
    c+_idx1 c+_idx2 of the environment chain, carried to length new_idx."""
    n1 = be.get_oper(1, 0, ch.env, ops["elec_up"], idx1, idx2, False, "F")
    n2 = be.get_oper(1, 0, ch.env, ops["elec_up"], idx2, idx2, False, "F")
    new = be.block_mul_block_ndia(n1, "N", n2, "N", 1.0, 0, ch.env_bases[idx2])
    env = be.update_trun(0, new, ch.env_truns[idx2]) if idx2 > ch.trun_idx else new
    return be.change_oper(1, 0, ch.env, env, idx2, new_idx, truns, "B")


def pairing_cor(be, ch: Chains, wave, ops, neib, xc1: int, xc2: int, ij: int, ny: int,
                num_site: int) -> Dict[Tuple[int, int, int], float]:
    """Get_mSCOP_Operator_Cor0(wave, trun_idx, 'S0', ..., xc1, xc2, ij, ij1)
    (measure.f90:3377-3507): the singlet pair correlation <D+_(sid1,sid2)
    D_(sid3,sid4)> for the bond (sid1, sid2 = neib(sid1, ij)) and the bonds
    (sid3, sid4 = neib(sid3, j)), j = 1, 3, 5, of the sites sid3 of sid1's
    row, in the system block (four operators of one block) and in the
    environment block (a pair on each side).  neib(i, k) is the lattice's
    neighbour table.  Returns {(sid1, sid3, j): value}; the reference's file
    output and its column of disconnected products are left out."""
    sys_len, env_len = ch.sys_len, ch.env_len
    sys_bs, env_bs = ch.sys_bases[sys_len], ch.env_bases[env_len]
    out = {}

    def env_part(sid1, sid2, sys_oper, sid3_range):
        for sid3 in sid3_range:
            if (sid3 - sid1) % ny != 0:
                continue
            eid1 = num_site - sid3 + 1
            for j in (1, 3, 5):
                sid4 = int(neib(sid3, j))
                eid2 = num_site - sid4 + 1
                if max(eid1, eid2) <= env_len - 1:
                    env_oper = get_scop_operator_env(be, ch, min(eid1, eid2), max(eid1, eid2), env_len - 1, True, ops)
                    out[(sid1, sid3, j)] = be.correlator("sys_block_env_block_cor_ndia", sys_oper, env_oper, sys_bs,
                                                         env_bs, wave, "B")

    for sid11 in range(xc1, xc2 + 1, ny):
        sid1 = sid11
        sid2 = int(neib(sid1, ij))
        pair = get_sys_two(be, ch, min(sid1, sid2), max(sid1, sid2), ops)
        for sid3 in range(sid1 + ny, sys_len - 3 + 1, ny):
            for j in (1, 3, 5):
                sid4 = int(neib(sid3, j))
                if min(sid4, sid3) <= max(sid1, sid2):
                    continue
                if max(sid3, sid4) <= sys_len - 1:
                    four = get_sys_two1(be, ch, max(sid1, sid2), min(sid3, sid4), max(sid3, sid4), pair, ops)
                    out[(sid1, sid3, j)] = be.correlator("measure_sys_block", four, None, sys_bs, None, wave)
        if ny >= 6:
            s1 = sid11 + 4
            s2 = int(neib(s1, ij))
            p1 = get_sys_two(be, ch, min(s1, s2), max(s1, s2), ops)
            sys_oper = be.change_oper(0, 0, ch.sys, p1, s2, sys_len - 1, True, "B")
            env_part(s1, s2, sys_oper, range(sys_len + 2, sys_len + ny + 2))
        sys_oper = be.change_oper(0, 0, ch.sys, pair, sid2, sys_len - 1, True, "B")
        env_part(sid1, sid2, sys_oper, range(sys_len + 2, num_site - ny + 1))
    return out


def measurement(be, dmrg, ops=None) -> Dict[str, Dict[tuple, float]]:
    """The correlator part of Measurement (main.f90:191-332) for the
    wavefunction `dmrg.wave` left by Get_Ground_State's last half-sweep: the
    reference site xc1 = (Nx / 6) ny - ny + 1, then
      pair_y  Get_mSCOP_Operator_Cor0(..., 'S0', xc1, xc1, 1, 0)  (main.f90:257)
      pair_x  Get_mSCOP_Operator_Cor0(..., 'S0', xc1, xc1, 3, 0)  (main.f90:258)
      density Get_density_cor(num_elec, num_elec, 'B', xc1)        (main.f90:274)
      spin    Get_density_cor(st_sd, st_sd, 'B', xc1)              (main.f90:286)
      elec    Get_density_cor(st_elec_up, st_elec_down, 'F', xc1)  (main.f90:299)
    each as {site tuple: value}; the files the reference writes are left out."""
    from .sweep import site_block_ops
    geo, wave = dmrg.geo, dmrg.wave
    ops = site_block_ops(dmrg.up_bias) if ops is None else ops
    ny, n = geo.ny, dmrg.N
    xc1 = (geo.nx // 6) * ny - ny + 1
    ch = Chains(dmrg, wave)
    geo.setup(wave.sys_len - 1, wave.env_len - 1)
    neib_tab = geo.neib.copy()

    def neib(i, k):
        return int(neib_tab[i, k])

    return {
        "pair_y": pairing_cor(be, ch, wave, ops, neib, xc1, xc1, 1, ny, n),
        "pair_x": pairing_cor(be, ch, wave, ops, neib, xc1, xc1, 3, ny, n),
        "density": density_cor(be, ch, wave, ops["num_elec"], ops["num_elec"], "B", xc1, ny, n),
        "spin": density_cor(be, ch, wave, ops["st_sd"], ops["st_sd"], "B", xc1, ny, n),
        "elec": density_cor(be, ch, wave, ops["elec_up"], ops["elec_down"], "F", xc1, ny, n),
    }
