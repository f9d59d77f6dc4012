"""Standalone two-site SU(2) DMRG driver over the hot-path entry points.

The reference's sweep driver is Fortran (code/tjsq/dmrg_sub.f90:553-1087:
warm_up_point, left_to_right, right_to_left, with main.f90:96-187 setting
the schedule); in a drop-in use it stays the caller of this library.  This
module restates it so that the library can be driven end to end without
the Fortran: the same block growth, the same targets, the same order of
calls -- Lanczos, density matrix and truncation, operator renormalisation,
wavefunction prediction -- with the blocks, truncations and bases kept in
memory where the reference writes them to disk (model_to_disk /
truns_to_disk / basis_to_disk, block.f90:2760-3097).

Every hot-path call goes through a backend object with the methods

  lanczos(lat, sys, env, sys_bs, env_bs, wave, lanzero) -> (E0, iters, wave)
  truncation(wave, side, kept_min, kept_max, trun_err) -> (info, trun Block)
  get_hamiltonian(lat, side, mshift, pre, basis, trun) -> Model
  wave_trans(direction, sys_bs, env_bs, sys_trun, env_trun, old, new_wave) -> new_wave

`DeviceBackend` (grand_sql_tj_b200.lib) runs them on the B200 through the C
ABI.
"""
from __future__ import annotations

import math
import time
from dataclasses import dataclass, field
from typing import Dict, List, Optional

import numpy as np

from .lattice import Geometry
from .structs import Basis, Block, BlockSet, Model, SubBlock, Wave
from .synth import get_basis, get_super_basis, site_sectors


def site_block_ops(up_bias: int) -> Dict[str, Block]:
    """Site operators of Get_site_operator_su2_U0 (dmrg_sub.f90:370-473)."""
    f = lambda v: np.full((1, 1), v, order="F")
    eu = Block(1, up_bias, 1, [SubBlock(0, 0, 1, f(-math.sqrt(2.0)))])
    ed = Block(1, -up_bias, 1, [SubBlock(up_bias, 1, -1, f(-math.sqrt(2.0)))])
    ne = Block(1, 0, 0, [SubBlock(0, 0, 0, f(0.0)), SubBlock(up_bias, 1, 0, f(math.sqrt(2.0)))])
    sd = Block(1, 0, 2, [SubBlock(up_bias, 1, 0, f(math.sqrt(1.5)))])
    return {"elec_up": eu, "elec_down": ed, "num_elec": ne, "st_sd": sd}


def site_model(up_bias: int, esite: float) -> Model:
    """Get_hamiltonian_site (dmrg_sub.f90:478-520) with the on-site energy
    esite * num_elec in the Hamiltonian (dmrg_sub.f90:578-590)."""
    o = site_block_ops(up_bias)
    ham = Block(1, 0, 0, [SubBlock(s.num_up, s.num_down, 0, np.asfortranarray(esite * s.mat)) for s in o["num_elec"].subs])
    sets = BlockSet(o["elec_up"], o["elec_down"], o["st_sd"], Block(1, 0, 0, []), o["num_elec"])
    return Model(1, ham, [sets])


def block_sectors_of(m: Model):
    """(num_up, num_down, dim) of the block's sectors, in its Hamiltonian's order (Get_basis reads ham)."""
    return [(s.num_up, s.num_down, s.mat.shape[1]) for s in m.ham.subs]


def identity_trun(bs: Basis) -> Block:
    """block_transfer_basis with unit matrices (dmrg_sub.f90:659-667): the
    warm-up's truncation while the enlarged block holds <= kept_max states."""
    return Block(bs.len, 0, 0, [SubBlock(m.new_num_up, m.new_num_down, 0, np.asfortranarray(np.eye(m.dim)))
                                for m in bs.maps])


def wave_initialize(wave: Wave, rng) -> None:
    """wave_initialize (block.f90:2437-2450): uniform [0, 1) entries sector by
    sector, then normalised; the reference's generator is Fortran's
    random_number with no seed, here a seeded numpy generator."""
    wave.data[:wave.dim] = rng.random(wave.dim)
    wave.data[:wave.dim] /= np.linalg.norm(wave.data[:wave.dim])


@dataclass
class StepRecord:
    phase: str
    sys_len: int
    env_len: int
    energy: float
    iters: int
    dim: int
    trunc_err: float = 0.0
    num_state: int = 0
    seconds: float = 0.0
    t_lanczos: float = 0.0
    t_trunc: float = 0.0
    t_renorm: float = 0.0
    t_pred: float = 0.0


@dataclass
class LastSuperblock:
    lat: object
    sys: Model
    env: Model
    sys_bs: Basis
    env_bs: Basis
    wave: Wave


@dataclass
class DmrgParams:
    n_elec: int                  # tot_num_up of the canonical run (up_bias = 1); 0 when grand-canonical
    tot_num_down: int = 0        # twice the target total spin
    kept_min: int = 64
    kept_max: int = 128
    trun_err: float = 1.0e-18
    lanzero: float = 2.0e-5      # Lanczos stop threshold of the sweeps (main.f90:169)
    lanzero_warm: float = 2.0e-2  # warm-up threshold, lanerr*10**3 (main.f90:104)
    seed: int = 1


class Dmrg:
    """Two-site DMRG of an Nx x Ny t-J cylinder, as the reference runs it."""

    def __init__(self, geo: Geometry, backend, p: DmrgParams):
        self.geo, self.be, self.p = geo, backend, p
        self.rng = np.random.default_rng(p.seed)
        self.up_bias = geo.up_bias
        self.N = geo.num_site
        self.sysblocks: Dict[int, Model] = {}
        self.envblocks: Dict[int, Model] = {}
        self.systruns: Dict[int, Block] = {}
        self.envtruns: Dict[int, Block] = {}
        self.sysbs: Dict[int, Basis] = {}
        self.envbs: Dict[int, Basis] = {}
        self.wave: Optional[Wave] = None
        self.last: Optional[LastSuperblock] = None
        self.records: List[StepRecord] = []
        self.site = site_sectors(self.up_bias)

    # ------------------------------------------------------------ helpers
    def _basis(self, m: Model) -> Basis:
        return get_basis(block_sectors_of(m), self.site, m.len + 1)

    def _trunc(self, wave: Wave, side: int, bs: Basis, kept_min: int, kept_max: int, trun_err: float,
               identity_below: bool):
        if identity_below and bs.dim <= kept_max:
            return identity_trun(bs), 0.0, bs.dim
        info, trun = self.be.truncation(wave, side, kept_min, kept_max, trun_err)
        return trun, float(info.trunc_err), int(info.num_state)

    def _lanczos(self, lat, sys, env, sys_bs, env_bs, wave, lanzero):
        e, it, w = self.be.lanczos(lat, sys, env, sys_bs, env_bs, wave, lanzero)
        # the superblock of the last step (its models, bases and ground state)
        self.last = LastSuperblock(lat, sys, env, sys_bs, env_bs, w)
        return e, it, w

    # ------------------------------------------------------------ warm-up
    def warm_up(self, end_id: Optional[int] = None, lanzero: Optional[float] = None,
                trun_err: Optional[float] = None) -> List[StepRecord]:
        """warm_up_point(bg_id = 1, end_id, ...) (dmrg_sub.f90:553-727):
        infinite-size growth of both blocks from single sites, truncating
        each enlarged block once it holds more than kept_max states."""
        p, geo = self.p, self.geo
        end_id = self.N // 2 if end_id is None else end_id
        lanzero = p.lanzero_warm if lanzero is None else lanzero
        trun_err = p.trun_err * 200 if trun_err is None else trun_err
        label = 1
        sys = site_model(self.up_bias, float(geo.esite[1]))
        env = site_model(self.up_bias, float(geo.esite[self.N]))
        self.sysblocks[1], self.envblocks[1] = sys, env
        out = []
        while label + 1 <= end_id:
            t0 = time.perf_counter()
            sys_bs, env_bs = self._basis(sys), self._basis(env)
            lat = geo.lattice(sys.len, env.len)
            tot_up = int(1.0 * (sys_bs.len + env_bs.len) / self.N * p.n_elec + 0.001)
            tot_down = int((p.tot_num_down * 1.0 / self.N) * (sys_bs.len + env_bs.len) + 0.5)
            tot_up -= tot_up % 2
            tot_up = min(tot_up, p.n_elec)
            tot_down = min(tot_down, p.tot_num_down)
            secs = get_super_basis(sys_bs, env_bs, tot_up if self.up_bias else 0, tot_down)
            wave = Wave(sys_bs.len, env_bs.len, secs)
            wave_initialize(wave, self.rng)
            e, it, wave = self._lanczos(lat, sys, env, sys_bs, env_bs, wave, lanzero)
            t1 = time.perf_counter()
            strun, serr, sn = self._trunc(wave, 0, sys_bs, p.kept_min, p.kept_max, trun_err, True)
            etrun, _, _ = self._trunc(wave, 1, env_bs, p.kept_min, p.kept_max, trun_err, True)
            t2 = time.perf_counter()
            sys = self.be.get_hamiltonian(lat, 0, 0, sys, sys_bs, strun)
            env = self.be.get_hamiltonian(lat, 1, sys.len, env, env_bs, etrun)
            t3 = time.perf_counter()
            self.sysblocks[label + 1], self.envblocks[label + 1] = sys, env
            self.systruns[label + 1], self.envtruns[label + 1] = strun, etrun
            self.sysbs[label + 1], self.envbs[label + 1] = sys_bs, env_bs
            self.wave = wave
            r = StepRecord("warmup", sys_bs.len - 1, env_bs.len - 1, e, it, wave.dim, serr, sn,
                           t3 - t0, t1 - t0, t2 - t1, t3 - t2)
            out.append(r)
            self.records.append(r)
            label += 1
        return out

    # ------------------------------------------------------------ sweeps
    def _start_wave(self, secs, sys_len, env_len, restart: bool, direction: int, trans_args):
        """The initial vector of a sweep's first step (dmrg_sub.f90:763-788 /
        945-971): random for a fresh start, else the last step's vector, carried
        to this superblock when its lengths differ."""
        new = Wave(sys_len, env_len, secs)
        if not restart or self.wave is None:
            wave_initialize(new, self.rng)
            return new
        if self.wave.sys_len != sys_len:
            return self.be.wave_trans(direction, *trans_args(), self.wave, new)
        new.data[:new.dim] = self.wave.data[:self.wave.dim]
        return new

    def left_to_right(self, bg_id: int, end_id: int, restart: bool = True, lanzero: Optional[float] = None,
                      trun_err: Optional[float] = None, phase: str = "L->R") -> List[StepRecord]:
        """left_to_right (dmrg_sub.f90:729-907): the system block grows from
        length bg_id to end_id - 1 + 1, each step truncated by its density
        matrix, the wavefunction carried from step to step by wave_trans_LR."""
        p, geo, N = self.p, self.geo, self.N
        lanzero = p.lanzero if lanzero is None else lanzero
        trun_err = p.trun_err if trun_err is None else trun_err
        tot_up = p.n_elec if self.up_bias else 0
        label = bg_id
        sys = self.sysblocks[label]
        env = self.envblocks[N - label - 2]
        out = []
        sys_trun = None
        first = True
        while first or label + 1 <= end_id:
            t0 = time.perf_counter()
            lat = geo.lattice(sys.len, env.len)
            sys_bs = self._basis(sys)
            env_bs = self._basis(env) if first else self.envbs[N - label - 1]
            secs = get_super_basis(sys_bs, env_bs, tot_up, p.tot_num_down)
            if first:
                wave = self._start_wave(secs, sys_bs.len, env_bs.len, restart, 0,
                                        lambda: (sys_bs, self.envbs[N - label], self.systruns[label],
                                                 self.envtruns[N - label - 1]))
            else:
                wave = self.be.wave_trans(0, sys_bs, self.envbs[N - label], sys_trun, self.envtruns[N - label - 1],
                                          self.wave, Wave(sys_bs.len, env_bs.len, secs))
            tp = time.perf_counter()
            e, it, wave = self._lanczos(lat, sys, env, sys_bs, env_bs, wave, lanzero)
            t1 = time.perf_counter()
            info, sys_trun = self.be.truncation(wave, 0, p.kept_min, p.kept_max, trun_err)
            t2 = time.perf_counter()
            sys = self.be.get_hamiltonian(lat, 0, 0, sys, sys_bs, sys_trun)
            t3 = time.perf_counter()
            self.sysblocks[label + 1], self.systruns[label + 1], self.sysbs[label + 1] = sys, sys_trun, sys_bs
            self.wave = wave
            r = StepRecord(phase, sys_bs.len - 1, env_bs.len - 1, e, it, wave.dim, float(info.trunc_err),
                           int(info.num_state), t3 - t0, t1 - tp, t2 - t1, t3 - t2, tp - t0)
            out.append(r)
            self.records.append(r)
            label += 1
            first = False
            if label + 1 <= end_id:
                env = self.envblocks[N - label - 2]
        return out

    def right_to_left(self, bg_id: int, end_id: int, restart: bool = True, lanzero: Optional[float] = None,
                      trun_err: Optional[float] = None, phase: str = "R->L") -> List[StepRecord]:
        """right_to_left (dmrg_sub.f90:911-1087): the environment block grows
        while the system block shrinks from length bg_id - 1 to end_id - 1,
        the wavefunction carried by wave_trans_RL."""
        p, geo, N = self.p, self.geo, self.N
        lanzero = p.lanzero if lanzero is None else lanzero
        trun_err = p.trun_err if trun_err is None else trun_err
        tot_up = p.n_elec if self.up_bias else 0
        label = bg_id
        sys = self.sysblocks[label - 1]
        env = self.envblocks[N - label - 1]
        out = []
        env_trun = None
        first = True
        while first or label - 1 >= end_id:
            t0 = time.perf_counter()
            lat = geo.lattice(sys.len, env.len)
            sys_bs = self._basis(sys) if first else self.sysbs[label]
            env_bs = self._basis(env)
            secs = get_super_basis(sys_bs, env_bs, tot_up, p.tot_num_down)
            if first:
                wave = self._start_wave(secs, sys_bs.len, env_bs.len, restart, 1,
                                        lambda: (self.sysbs[label + 1], env_bs, self.systruns[label],
                                                 self.envtruns[N - label - 1]))
            else:
                wave = self.be.wave_trans(1, self.sysbs[label + 1], env_bs, self.systruns[label], env_trun,
                                          self.wave, Wave(sys_bs.len, env_bs.len, secs))
            tp = time.perf_counter()
            e, it, wave = self._lanczos(lat, sys, env, sys_bs, env_bs, wave, lanzero)
            t1 = time.perf_counter()
            info, env_trun = self.be.truncation(wave, 1, p.kept_min, p.kept_max, trun_err)
            t2 = time.perf_counter()
            env = self.be.get_hamiltonian(lat, 1, sys.len + 1, env, env_bs, env_trun)
            t3 = time.perf_counter()
            self.envblocks[N - label], self.envtruns[N - label], self.envbs[N - label] = env, env_trun, env_bs
            self.wave = wave
            r = StepRecord(phase, sys_bs.len - 1, env_bs.len - 1, e, it, wave.dim, float(info.trunc_err),
                           int(info.num_state), t3 - t0, t1 - tp, t2 - t1, t3 - t2, tp - t0)
            out.append(r)
            self.records.append(r)
            label -= 1
            first = False
            if label - 1 >= end_id:
                sys = self.sysblocks[label - 1]
        return out

    def ground_state(self, sweeps: int, final_half: bool = False) -> List[StepRecord]:
        """Get_Ground_State (main.f90:96-187) for a fresh start: warm-up to
        half the lattice, a left-to-right half-sweep from a random vector, a
        right-to-left half-sweep, then `sweeps` full sweeps (left to right and
        back) at the sweep thresholds; kept_max and the thresholds as given in
        the parameters (the reference's kept-state schedule is left to the
        caller)."""
        N = self.N
        self.warm_up()
        self.left_to_right(N // 2 - 1, N - 2, restart=False, phase="L->R0")
        self.right_to_left(N - 2, 1, restart=True, phase="R->L0")
        for s in range(sweeps):
            self.left_to_right(1, N - 2, restart=True, phase="L->R%d" % (s + 1))
            self.right_to_left(N - 2, 1, restart=True, phase="R->L%d" % (s + 1))
        if final_half:
            self.left_to_right(1, N // 2 + 3, restart=True, phase="final")
        return self.records
