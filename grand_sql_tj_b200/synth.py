"""Seeded synthetic superblocks with the structure of a tjsq DMRG step.

No DMRG run of the reference can be reproduced here (no Fortran compiler, and
a 4x24 m=2000 sweep takes days on a CPU), so benchmark and test inputs are
built directly: block sector tables with a realistic spread of (N, 2S) labels
and multiplet counts, the enlarged bases and super basis exactly as the
reference builds them (Get_basis / Get_super_basis, block.f90:9-161), and
random operator blocks with the reference's quantum-number structure:

  ham, num_sn   down_dif 0, symmetric sector-diagonal blocks
  elec_up       c^+  : (N, 2S) -> (N + up_bias, 2S +- 1)
  elec_down     c    : (N, 2S) -> (N - up_bias, 2S +- 1)
  spin_sd       S    : (N, 2S) -> (N, 2S + {-2, 0, 2}) with the reduced
                       Hermiticity <s||S||t> = (-1)^((s-t)/2) <t||S||s>

The last rule and symmetric ham/num_sn make H*psi a symmetric operator, as
it is for a real DMRG block (checked by the test-suite).
"""
from __future__ import annotations

import math
from dataclasses import dataclass
from typing import Dict, List, Optional, Sequence, Tuple

import numpy as np

from .lattice import Geometry
from .structs import (Basis, BasisMap, Block, BlockSet, Lattice, Model, SubBlock, Wave,
                      WaveSector)

Sector = Tuple[int, int, int]   # (num_up, num_down, dim)


def site_sectors(up_bias: int) -> List[Sector]:
    """Sectors of the single-site operator st_sz used by Get_basis (dmrg_sub.f90:444-466)."""
    return [(0, 0, 1), (up_bias, 1, 1)]


def _sort_qn_desc(pairs):
    # QuickSort_Integer (block.f90:206-239): descending in num_down, then in num_up
    return sorted(pairs, key=lambda p: (-p[1], -p[0]))


def get_basis(block: Sequence[Sector], site: Sequence[Sector], length: int) -> Basis:
    """Get_basis (block.f90:9-104): block (x) site -> enlarged block."""
    pre = []
    for (bu, bd, _) in block:
        for (su, sd, _) in site:
            for ss in range(abs(bd - sd), bd + sd + 1, 2):
                pre.append((bu + su, ss))
    uniq = []
    for p in _sort_qn_desc(pre):
        if not uniq or uniq[-1] != p:
            uniq.append(p)
    maps = []
    for (nu, nd) in uniq:
        subs, pos = [], 0
        for (bu, bd, bdim) in block:
            for (su, sd, sdim) in site:
                if bu + su == nu and abs(bd - sd) <= nd <= bd + sd:
                    subs.append((pos, bdim * sdim, bu, bd, su, sd))
                    pos += bdim * sdim
        maps.append(BasisMap(nu, nd, subs))
    return Basis(length, maps)


def get_super_basis(sys_bs: Basis, env_bs: Basis, total_up: int, total_down: int) -> List[WaveSector]:
    """Get_super_basis (block.f90:110-161)."""
    out = []
    for x in sys_bs.maps:
        for y in env_bs.maps:
            if y.new_num_up == total_up - x.new_num_up:
                if abs(y.new_num_down - x.new_num_down) <= total_down <= y.new_num_down + x.new_num_down:
                    out.append(WaveSector(x.new_num_up, x.new_num_down, y.new_num_up, y.new_num_down,
                                          x.dim, y.dim))
    return out


def block_sectors(m: int, n_center: float, up_bias: int, sigma_n: float = 2.2,
                  s_weights: Sequence[float] = (1.0, 1.0, 0.8, 0.55, 0.3, 0.14, 0.06, 0.025, 0.01),
                  max_sector: Optional[int] = None) -> List[Sector]:
    """Multiplet counts of a renormalised block keeping m multiplets.

    Canonical labels (up_bias = 1): (N, 2S) with 2S = N mod 2, weight
    exp(-(N-n_center)^2 / (2 sigma_n^2)) * s_weights[2S]; grand-canonical
    labels (up_bias = 0): (0, 2S) with weight s_weights[2S].
    """
    cand = []
    if up_bias:
        lo, hi = int(math.floor(n_center - 4 * sigma_n)), int(math.ceil(n_center + 4 * sigma_n))
        for n in range(max(lo, 0), hi + 1):
            for s2 in range(n % 2, len(s_weights), 2):
                w = math.exp(-(n - n_center) ** 2 / (2 * sigma_n ** 2)) * s_weights[s2]
                cand.append((n, s2, w))
    else:
        for s2 in range(len(s_weights)):
            cand.append((0, s2, s_weights[s2]))
    tot = sum(c[2] for c in cand)
    secs = []
    for (n, s2, w) in cand:
        d = int(round(m * w / tot))
        if max_sector:
            d = min(d, max_sector)
        if d >= 1:
            secs.append((n, s2, d))
    return _sort_qn_desc(secs)


def _sym(rng, n, scale):
    a = rng.standard_normal((n, n)) * scale
    return np.asfortranarray((a + a.T) * 0.5)


def make_ops(secs: List[Sector], length: int, up_bias: int, nslots: int, rng,
             ham_spread: float = 4.0) -> Tuple[Block, List[BlockSet]]:
    """Hamiltonian and per-site operator sets of one block."""
    idx: Dict[Tuple[int, int], int] = {(s[0], s[1]): k for k, s in enumerate(secs)}
    dims = {(s[0], s[1]): s[2] for s in secs}
    ham_subs = []
    for (nu, nd, d) in secs:
        e = np.sort(rng.uniform(-ham_spread, ham_spread, d))
        h = np.diag(e) + _sym(rng, d, 0.3 / math.sqrt(d))
        ham_subs.append(SubBlock(nu, nd, 0, np.asfortranarray(h)))
    ham = Block(length, 0, 0, ham_subs)

    def gen_sets():
        eu, ed, sd, sn = [], [], [], []
        for (nu, nd, d) in secs:
            for dd in (-1, 1):
                t = (nu + up_bias, nd + dd)
                if nd + dd >= 0 and t in dims:
                    eu.append(SubBlock(nu, nd, dd, np.asfortranarray(rng.standard_normal((dims[t], d)) / math.sqrt(d))))
            for dd in (-1, 1):
                t = (nu - up_bias, nd + dd)
                if nd + dd >= 0 and t in dims:
                    ed.append(SubBlock(nu, nd, dd, np.asfortranarray(rng.standard_normal((dims[t], d)) / math.sqrt(d))))
            sn.append(SubBlock(nu, nd, 0, _sym(rng, d, 1.0 / math.sqrt(d))))
        # spin_sd with the reduced Hermiticity relation
        pair: Dict[Tuple[int, int, int], np.ndarray] = {}
        for (nu, nd, d) in secs:
            for dd in (-2, 0, 2):
                t = (nu, nd + dd)
                if nd + dd < 0 or t not in dims or (dd == 0 and nd == 0):
                    continue
                if dd == 0:
                    pair[(nu, nd, 0)] = _sym(rng, d, 1.0 / math.sqrt(d))
                elif dd == 2:
                    pair[(nu, nd, 2)] = np.asfortranarray(rng.standard_normal((dims[t], d)) / math.sqrt(d))
        for (nu, nd, d) in secs:
            for dd in (-2, 0, 2):
                t = (nu, nd + dd)
                if nd + dd < 0 or t not in dims or (dd == 0 and nd == 0):
                    continue
                if dd == -2:
                    m = -pair[(nu, nd - 2, 2)].T
                else:
                    m = pair[(nu, nd, dd)]
                sd.append(SubBlock(nu, nd, dd, np.asfortranarray(m)))
        return BlockSet(Block(length, up_bias, 1, eu), Block(length, -up_bias, 1, ed),
                        Block(length, 0, 2, sd), Block(length, 0, 0, []), Block(length, 0, 0, sn))

    return ham, [gen_sets() for _ in range(nslots)]


@dataclass
class Superblock:
    geo: Geometry
    lat: Lattice
    sys: Model
    env: Model
    sys_bs: Basis
    env_bs: Basis
    wave: Wave
    tot_num_up: int
    sys_secs: List[Sector]
    env_secs: List[Sector]

    def flops_hint(self) -> float:
        return float(self.wave.dim)


def make_superblock(nx: int, ny: int, sys_len: int, env_len: int, m: int, n_elec: int,
                    seed: int, up_bias: int = 1, t: float = 1.0, J: float = 1.0 / 3.0,
                    t2: float = 0.0, esite: float = -0.7, sigma_n: float = 2.2,
                    s_weights: Optional[Sequence[float]] = None,
                    max_sector: Optional[int] = None) -> Superblock:
    """One two-site superblock [sys_len + 2 sites + env_len] of an nx x ny cylinder."""
    rng = np.random.default_rng(seed)
    geo = Geometry(nx, ny, t=t, J=J, t2=t2, esite=esite, up_bias=up_bias)
    lat = geo.lattice(sys_len, env_len)
    n_site = nx * ny
    kw = {} if s_weights is None else {"s_weights": s_weights}
    ncs = n_elec * sys_len / n_site
    nce = n_elec * env_len / n_site
    ssec = block_sectors(m, ncs, up_bias, sigma_n=sigma_n, max_sector=max_sector, **kw)
    esec = block_sectors(m, nce, up_bias, sigma_n=sigma_n, max_sector=max_sector, **kw)
    site = site_sectors(up_bias)
    sys_bs = get_basis(ssec, site, sys_len + 1)
    env_bs = get_basis(esec, site, env_len + 1)
    tot_up = n_elec if up_bias else 0
    secs = get_super_basis(sys_bs, env_bs, tot_up, 0)
    nss = int(geo.nleg11[sys_len - 1])
    nse = int(geo.nleg11[env_len - 1])
    sham, ssets = make_ops(ssec, sys_len, up_bias, nss, rng)
    eham, esets = make_ops(esec, env_len, up_bias, nse, rng)
    wave = Wave(sys_len + 1, env_len + 1, secs)
    # wave_initialize (block.f90:2437-2450): uniform [0,1) entries, normalised
    wave.data[:] = rng.random(wave.data.shape[0])
    wave.data /= np.linalg.norm(wave.data)
    return Superblock(geo, lat, Model(sys_len, sham, ssets), Model(env_len, eham, esets),
                      sys_bs, env_bs, wave, tot_up, ssec, esec)


# Named workloads ------------------------------------------------------------
def workload(name: str, seed: int = 1234) -> Superblock:
    """Superblocks of the benchmark configurations (and small test cases)."""
    if name == "tiny":        # 2x4 ladder, everything exercised, oracle in milliseconds
        return make_superblock(4, 2, 3, 3, 6, 6, seed, max_sector=4)
    if name == "small":       # 2x6 ladder
        return make_superblock(6, 2, 5, 5, 24, 10, seed)
    if name == "small_gc":    # grand-canonical labels (the shipped reference mode)
        return make_superblock(6, 2, 5, 5, 24, 0, seed, up_bias=0)
    if name == "cyl4":        # 4x6 cylinder, periodic in y
        return make_superblock(6, 4, 11, 11, 64, 20, seed)
    if name == "ladder16_m256":   # 2x16 ladder, 4 holes, m=256 (CPU-runnable configuration)
        return make_superblock(16, 2, 15, 15, 256, 28, seed)
    if name == "cyl4x24_m2000":   # 4x24 cylinder, 12 holes, m=2000, mid-chain superblock
        return make_superblock(24, 4, 47, 47, 2000, 84, seed)
    if name == "cyl4x24_m500":
        return make_superblock(24, 4, 47, 47, 500, 84, seed)
    if name == "cyl6x24_m6000":   # 6x24 cylinder, t'=-0.2, 18 holes, m=6000
        return make_superblock(24, 6, 71, 71, 6000, 126, seed, t2=-0.2)
    raise KeyError(name)


@dataclass
class RenormCase:
    """Inputs of one operator renormalisation (Get_Hamiltonian_Sys/Env)."""
    lat: Lattice
    side: int
    mshift: int
    pre: Model
    basis: Basis
    trun: Block


def random_trun(basis: Basis, kept: int, rng) -> Block:
    """A truncation operator keeping about `kept` states of `basis`: per sector
    a column-orthonormal matrix (row_dim = the sector's dimension) with the
    sector's share of the kept states (at least one)."""
    subs = []
    for m in basis.maps:
        k = max(1, min(m.dim, int(round(kept * m.dim / basis.dim))))
        q, _ = np.linalg.qr(rng.standard_normal((m.dim, k)))
        subs.append(SubBlock(m.new_num_up, m.new_num_down, 0, np.asfortranarray(q)))
    return Block(basis.len, 0, 0, subs)


def renorm_case(name: str, side: int = 0, seed: int = 1234) -> RenormCase:
    """The renormalisation of the system (side 0) or environment (side 1)
    block of a named superblock: the block is enlarged by its centre site and
    truncated back to about m states."""
    sb = workload(name, seed=seed)
    rng = np.random.default_rng(seed + 17)
    ms = {"tiny": 6, "small": 24, "small_gc": 24, "cyl4": 64, "ladder16_m256": 256, "cyl4x24_m2000": 2000,
          "cyl4x24_m500": 500, "cyl6x24_m6000": 6000}[name]
    pre = sb.sys if side == 0 else sb.env
    basis = sb.sys_bs if side == 0 else sb.env_bs
    trun = random_trun(basis, ms, rng)
    mshift = 0 if side == 0 else sb.sys.len + 1
    return RenormCase(sb.lat, side, mshift, pre, basis, trun)
