"""ctypes mirrors of the C ABI in include/tj_b200.h and a numpy-side data model.

The reference (code/tjsq/common.f90:65-149) keeps its block-sparse objects in
Fortran derived types.  This module holds the same objects as plain Python
classes backed by numpy arrays (column-major sub-matrices, as in Fortran) and
packs them into the flat C structs the library takes.  A packed object keeps
references to every numpy buffer it points into, so the pointers stay valid
for as long as the packed object lives.
"""
from __future__ import annotations

import ctypes as C
import time
from dataclasses import dataclass, field
from collections.abc import Sequence
from typing import List, Optional, Tuple

import numpy as np

c_int32_p = C.POINTER(C.c_int32)
c_double_p = C.POINTER(C.c_double)


class TjBlockSub(C.Structure):
    _fields_ = [("num_up", C.c_int32), ("num_down", C.c_int32), ("down_dif", C.c_int32),
                ("row_dim", C.c_int32), ("sdim", C.c_int32), ("pad_", C.c_int32),
                ("off", C.c_int64)]


class TjBlock(C.Structure):
    _fields_ = [("len", C.c_int32), ("num", C.c_int32), ("dim", C.c_int32),
                ("up_dif", C.c_int32), ("down_dif", C.c_int32), ("pad_", C.c_int32),
                ("sub", C.POINTER(TjBlockSub)), ("data", c_double_p)]


class TjBlockSet(C.Structure):
    _fields_ = [("elec_up", TjBlock), ("elec_down", TjBlock), ("spin_sd", TjBlock),
                ("spin_sz", TjBlock), ("num_sn", TjBlock)]


class TjModel(C.Structure):
    _fields_ = [("len", C.c_int32), ("nsub", C.c_int32), ("ham", TjBlock),
                ("sub", C.POINTER(TjBlockSet))]


class TjBasisSub(C.Structure):
    _fields_ = [("spos", C.c_int32), ("sdim", C.c_int32), ("bl_num_up", C.c_int32),
                ("bl_num_down", C.c_int32), ("st_num_up", C.c_int32), ("st_num_down", C.c_int32)]


class TjBasisMap(C.Structure):
    _fields_ = [("idx", C.c_int32), ("num", C.c_int32), ("dim", C.c_int32),
                ("new_num_up", C.c_int32), ("new_num_down", C.c_int32), ("first", C.c_int32)]


class TjBasis(C.Structure):
    _fields_ = [("len", C.c_int32), ("num", C.c_int32), ("dim", C.c_int32), ("pad_", C.c_int32),
                ("sub", C.POINTER(TjBasisMap)), ("maps", C.POINTER(TjBasisSub))]


class TjWaveSub(C.Structure):
    _fields_ = [("sys_num_up", C.c_int32), ("sys_num_down", C.c_int32),
                ("env_num_up", C.c_int32), ("env_num_down", C.c_int32),
                ("sys_dim", C.c_int32), ("env_dim", C.c_int32), ("off", C.c_int64)]


class TjWave(C.Structure):
    _fields_ = [("sys_len", C.c_int32), ("env_len", C.c_int32), ("num", C.c_int32),
                ("pad_", C.c_int32), ("dim", C.c_int64), ("sub", C.POINTER(TjWaveSub)),
                ("data", c_double_p)]


class TjLattice(C.Structure):
    _fields_ = [("num_site", C.c_int32), ("neibt", C.c_int32), ("up_bias", C.c_int32),
                ("pad_", C.c_int32),
                ("neib", c_int32_p), ("neiba", c_int32_p), ("inb1", c_int32_p),
                ("nleg11", c_int32_p), ("nposi", c_int32_p), ("nposi_dm", c_int32_p),
                ("nposi_lat", c_int32_p),
                ("jt", c_double_p), ("jz", c_double_p), ("jd", c_double_p), ("jn", c_double_p),
                ("esite", c_double_p)]


class TjTruncResult(C.Structure):
    _fields_ = [("num_state", C.c_int32), ("num", C.c_int32), ("data_len", C.c_int64),
                ("trunc_err", C.c_double), ("entropy1", C.c_double), ("entropy2", C.c_double),
                ("entropys", C.c_double), ("sub", C.POINTER(TjBlockSub)), ("data", c_double_p)]


class TjModelResult(C.Structure):
    _fields_ = [("len", C.c_int32), ("nsub", C.c_int32), ("n_subs", C.c_int32), ("pad_", C.c_int32),
                ("data_len", C.c_int64), ("sets", C.POINTER(TjBlockSet)), ("subs", C.POINTER(TjBlockSub)),
                ("data", c_double_p), ("model", TjModel)]


class TjBlockResult(C.Structure):
    _fields_ = [("num", C.c_int32), ("pad_", C.c_int32), ("data_len", C.c_int64),
                ("subs", C.POINTER(TjBlockSub)), ("data", c_double_p), ("block", TjBlock)]


class TjChain(C.Structure):
    _fields_ = [("n", C.c_int32), ("trun_idx", C.c_int32), ("bsm", C.POINTER(TjBasis)),
                ("truns", C.POINTER(TjBlock))]


class TjBasisResult(C.Structure):
    _fields_ = [("len", C.c_int32), ("num", C.c_int32), ("dim", C.c_int32), ("nmaps", C.c_int32),
                ("sub", C.POINTER(TjBasisMap)), ("maps", C.POINTER(TjBasisSub)), ("basis", TjBasis)]


class TjHpsiStats(C.Structure):
    _fields_ = [("flops", C.c_double), ("flops_ref", C.c_double), ("bytes", C.c_double),
                ("n_products", C.c_int64), ("n_tasks", C.c_int64), ("n_tiles_p1", C.c_int64),
                ("n_tiles_p2", C.c_int64), ("scratch_doubles", C.c_int64),
                ("last_ms", C.c_double), ("last_ms_phase1", C.c_double),
                ("last_ms_phase2", C.c_double), ("lanczos_hpsi", C.c_int64),
                ("int8_ops", C.c_double), ("kernels_per_hpsi", C.c_int64), ("last_ms_split", C.c_double),
                ("flops_launch1", C.c_double), ("flops_launch2", C.c_double),
                ("int8_ops_launch1", C.c_double), ("int8_ops_launch2", C.c_double),
                ("prepare_ms", C.c_double), ("plan_ms", C.c_double), ("upload_ms", C.c_double),
                ("ozplan_ms", C.c_double), ("lanczos_ms", C.c_double),
                ("renorm_plan_ms", C.c_double), ("renorm_ms", C.c_double), ("renorm_e2e_ms", C.c_double),
                ("renorm_flops", C.c_double),
                ("trunc_ms_rho", C.c_double), ("trunc_ms_tridiag", C.c_double), ("trunc_ms_eig", C.c_double),
                ("trunc_ms_select", C.c_double), ("trunc_ms_vec", C.c_double), ("trunc_ms_orth", C.c_double),
                ("trunc_ms_back", C.c_double), ("trunc_ms_total", C.c_double),
                ("trunc_max_n", C.c_int64), ("trunc_max_kept", C.c_int64),
                ("res_hits", C.c_int64), ("res_hit_bytes", C.c_double),
                ("renorm_pre_ms", C.c_double), ("renorm_post_ms", C.c_double),
                ("wt_plan_ms", C.c_double), ("wt_ms", C.c_double)]


class TjTuneResult(C.Structure):
    _fields_ = [(n, C.c_int32) for n in ("items_per_cta", "min_ksteps", "ctas_per_sm", "oz_bn", "oz_item_cost",
                                         "evaluated")] + \
               [("default_ms", C.c_double), ("tuned_ms", C.c_double), ("tuning_ms", C.c_double),
                ("hist_key", C.c_uint64)]

    def as_dict(self):
        return {n: getattr(self, n) for n, _ in self._fields_}


class TjGgCell(C.Structure):
    _fields_ = [("out_off", C.c_int64), ("M", C.c_int32), ("N", C.c_int32), ("t_begin", C.c_int32),
                ("t_end", C.c_int32)]


class TjGgTerm(C.Structure):
    _fields_ = [("l_off", C.c_int64), ("r_off", C.c_int64)] + \
               [(n, C.c_int32) for n in ("l_ld", "r_ld", "K", "l_trans", "r_trans", "pad_")] + \
               [("coef", C.c_double)]


def _dptr(a: np.ndarray):
    return a.ctypes.data_as(c_double_p)


def _iptr(a: np.ndarray):
    return a.ctypes.data_as(c_int32_p)


# --------------------------------------------------------------------------
# numpy-side objects
# --------------------------------------------------------------------------
@dataclass
class SubBlock:
    """Sub_Block: maps sector (num_up, num_down) by down_dif; mat is (row_dim, sdim)."""
    num_up: int
    num_down: int
    down_dif: int
    mat: np.ndarray


@dataclass
class Block:
    """Total_Block (common.f90:119-122)."""
    len: int
    up_dif: int
    down_dif: int
    subs: List[SubBlock] = field(default_factory=list)

    @property
    def dim(self) -> int:
        return int(sum(s.mat.shape[1] for s in self.subs))

    def pack(self) -> "PackedBlock":
        # a block the library returned keeps its result arrays: packed without
        # a copy while its sub-blocks are still those views
        pk = getattr(self, "_packed", None)
        return pk if pk is not None and pk.matches(self) else PackedBlock(self)


class _Views:
    """The sub-blocks of a block as made: the matrix objects themselves
    (held, so that an identity test cannot meet a recycled object) and
    their sector labels."""

    __slots__ = ("labels", "mats")

    def __init__(self, b: "Block"):
        self.labels = [(s.num_up, s.num_down, s.down_dif) for s in b.subs]
        self.mats = [s.mat for s in b.subs]

    def __eq__(self, other: "_Views") -> bool:
        return (len(self.mats) == len(other.mats) and all(a is b for a, b in zip(self.mats, other.mats))
                and self.labels == other.labels)


def _views(b: "Block") -> _Views:
    return _Views(b)


class _BlockView:
    """The packed form of a block the library wrote: its own sub-block table
    and data array (the sub-blocks of the Block are views into that array).
    It stands for the Block while every sub-block is still the view it was
    made with (matrices changed in place are seen through the views; a
    replaced sub-block makes pack() copy)."""

    def __init__(self, c, subs, data, block: "Block"):
        self.c, self.subs, self.data = c, subs, data
        self.views = _views(block)

    def matches(self, block: "Block") -> bool:
        return _views(block) == self.views


class PackedBlock:
    def __init__(self, b: Block):
        n = len(b.subs)
        self.subs = (TjBlockSub * max(n, 1))()
        total = int(sum(s.mat.size for s in b.subs))
        self.data = np.zeros(max(total, 1), dtype=np.float64)
        off = 0
        for i, s in enumerate(b.subs):
            r, c = s.mat.shape
            self.subs[i] = TjBlockSub(s.num_up, s.num_down, s.down_dif, r, c, 0, off)
            self.data[off:off + r * c] = np.asarray(s.mat, dtype=np.float64).reshape(-1, order="F")
            off += r * c
        self.c = TjBlock(b.len, n, b.dim, b.up_dif, b.down_dif, 0,
                         C.cast(self.subs, C.POINTER(TjBlockSub)), _dptr(self.data))


OPS = ("elec_up", "elec_down", "spin_sd", "spin_sz", "num_sn")


@dataclass
class BlockSet:
    elec_up: Block
    elec_down: Block
    spin_sd: Block
    spin_sz: Block
    num_sn: Block


@dataclass
class Model:
    """Total_Model inputs (common.f90:144-149): ham and sub(1:nsub)."""
    len: int
    ham: Block
    sub: List[BlockSet]

    def pack(self) -> "PackedModel":
        # a model the library returned keeps its result arrays: packed without
        # a copy while its blocks are still those views
        pk = getattr(self, "_packed", None)
        return pk if pk is not None and pk.matches(self) else PackedModel(self)


class PackedModel:
    def __init__(self, m: Model):
        self.ham = m.ham.pack()
        self.sets = []
        n = len(m.sub)
        self.sub = (TjBlockSet * max(n, 1))()
        for i, bs in enumerate(m.sub):
            ps = [getattr(bs, k).pack() for k in OPS]
            self.sets.append(ps)
            self.sub[i] = TjBlockSet(*[p.c for p in ps])
        self.c = TjModel(m.len, n, self.ham.c, C.cast(self.sub, C.POINTER(TjBlockSet)))


@dataclass
class BasisMap:
    new_num_up: int
    new_num_down: int
    # (spos, sdim, bl_num_up, bl_num_down, st_num_up, st_num_down)
    subs: List[Tuple[int, int, int, int, int, int]]

    @property
    def dim(self) -> int:
        return int(sum(s[1] for s in self.subs))


@dataclass
class Basis:
    """Total_Basis (common.f90:79-82)."""
    len: int
    maps: List[BasisMap]

    @property
    def dim(self) -> int:
        return int(sum(m.dim for m in self.maps))

    def pack(self) -> "PackedBasis":
        # a sweep passes each basis to several calls: the packed form is kept
        # while the maps read the same (comparing them costs a few
        # microseconds, packing a few hundred)
        sig = (self.len, [(m.new_num_up, m.new_num_down, tuple(m.subs)) for m in self.maps])
        pk = self.__dict__.get("_packed")
        if pk is None or pk[0] != sig:
            pk = (sig, PackedBasis(self))
            self.__dict__["_packed"] = pk
        return pk[1]


class PackedBasis:
    def __init__(self, b: Basis):
        n = len(b.maps)
        nm = sum(len(m.subs) for m in b.maps)
        self.sub = (TjBasisMap * max(n, 1))()
        self.maps = (TjBasisSub * max(nm, 1))()
        k = 0
        for i, m in enumerate(b.maps):
            self.sub[i] = TjBasisMap(0, len(m.subs), m.dim, m.new_num_up, m.new_num_down, k)
            for s in m.subs:
                self.maps[k] = TjBasisSub(*s)
                k += 1
        self.c = TjBasis(b.len, n, b.dim, 0, C.cast(self.sub, C.POINTER(TjBasisMap)),
                         C.cast(self.maps, C.POINTER(TjBasisSub)))


@dataclass
class WaveSector:
    sys_num_up: int
    sys_num_down: int
    env_num_up: int
    env_num_down: int
    sys_dim: int
    env_dim: int


class Wave:
    """Wavefunction (common.f90:100-110): sector matrices stored back to back."""

    def __init__(self, sys_len: int, env_len: int, sectors: List[WaveSector],
                 data: Optional[np.ndarray] = None):
        self.sys_len = sys_len
        self.env_len = env_len
        self.sectors = list(sectors)
        self.offsets = np.zeros(len(sectors) + 1, dtype=np.int64)
        for i, s in enumerate(sectors):
            self.offsets[i + 1] = self.offsets[i] + s.sys_dim * s.env_dim
        self.dim = int(self.offsets[-1])
        self.data = np.zeros(max(self.dim, 1), dtype=np.float64) if data is None else data
        assert self.data.dtype == np.float64 and self.data.flags.c_contiguous
        self.sub = (TjWaveSub * max(len(sectors), 1))()
        for i, s in enumerate(sectors):
            self.sub[i] = TjWaveSub(s.sys_num_up, s.sys_num_down, s.env_num_up, s.env_num_down,
                                    s.sys_dim, s.env_dim, int(self.offsets[i]))
        self.c = TjWave(sys_len, env_len, len(sectors), 0, self.dim,
                        C.cast(self.sub, C.POINTER(TjWaveSub)), _dptr(self.data))

    def like(self, data: Optional[np.ndarray] = None) -> "Wave":
        return Wave(self.sys_len, self.env_len, self.sectors,
                    np.zeros_like(self.data) if data is None else data)

    def copy(self) -> "Wave":
        return self.like(self.data.copy())

    def sector(self, i: int) -> np.ndarray:
        s = self.sectors[i]
        a = self.data[self.offsets[i]:self.offsets[i + 1]]
        return a.reshape((s.sys_dim, s.env_dim), order="F")


class Lattice:
    """Module pubdata globals read on the hot path, in the layouts of tj_lattice."""

    def __init__(self, num_site: int, neibt: int, up_bias: int, neib, neiba, inb1, nleg11,
                 nposi, nposi_dm, nposi_lat, jt, jz, jd, jn, esite):
        self.num_site, self.neibt, self.up_bias = num_site, neibt, up_bias
        ns1 = num_site + 1
        f = lambda a, shape: np.ascontiguousarray(np.asarray(a, dtype=np.int32).reshape(-1, order="F"))
        self.neib = f(neib, (ns1, neibt))
        self.neiba = f(neiba, (ns1, ns1))
        self.inb1 = f(inb1, (ns1, ns1))
        self.nleg11 = np.ascontiguousarray(np.asarray(nleg11, dtype=np.int32))
        self.nposi = np.ascontiguousarray(np.asarray(nposi, dtype=np.int32))
        self.nposi_dm = np.ascontiguousarray(np.asarray(nposi_dm, dtype=np.int32))
        self.nposi_lat = np.ascontiguousarray(np.asarray(nposi_lat, dtype=np.int32))
        d = lambda a: np.ascontiguousarray(np.asarray(a, dtype=np.float64).reshape(-1, order="F"))
        self.jt, self.jz, self.jd = d(jt), d(jz), d(jd)
        self.jn = d(jn)
        self.esite = d(esite)
        self.c = TjLattice(num_site, neibt, up_bias, 0, _iptr(self.neib), _iptr(self.neiba),
                           _iptr(self.inb1), _iptr(self.nleg11), _iptr(self.nposi),
                           _iptr(self.nposi_dm), _iptr(self.nposi_lat), _dptr(self.jt),
                           _dptr(self.jz), _dptr(self.jd), _dptr(self.jn), _dptr(self.esite))


def block_transfer_trans(b: Block) -> Block:
    """block_transfer_trans (block.f90:1676-1706): the transposed operator."""
    subs = [SubBlock(s.num_up + b.up_dif, s.num_down + s.down_dif, -s.down_dif, np.asfortranarray(s.mat.T))
            for s in b.subs]
    return Block(b.len, -b.up_dif, b.down_dif, subs)


# host wall time (s) of the stages of the last call_model_result
RESULT_HOST_S = {}


def call_model_result(call, alloc=None):
    """Runs a two-call model-result entry point `call(res_ptr) -> rc` and
    returns the new Model (views into its result arrays); alloc(n) gives the
    data array of n doubles (default: a new zeroed array)."""
    t0 = time.perf_counter()
    res = TjModelResult()
    rc = call(C.byref(res))
    if rc:
        return rc, None
    t1 = time.perf_counter()
    sets = (TjBlockSet * max(res.nsub, 1))()
    subs = (TjBlockSub * max(res.n_subs, 1))()
    data = np.zeros(max(res.data_len, 1)) if alloc is None else alloc(max(res.data_len, 1))
    res.sets = C.cast(sets, C.POINTER(TjBlockSet))
    res.subs = C.cast(subs, C.POINTER(TjBlockSub))
    res.data = data.ctypes.data_as(c_double_p)
    t2 = time.perf_counter()
    rc = call(C.byref(res))
    if rc:
        return rc, None
    t3 = time.perf_counter()
    m = model_from_c(res.model, data, keep=(res, sets, subs, data))
    RESULT_HOST_S.update(sizes=t1 - t0, alloc=t2 - t1, fill=t3 - t2, wrap=time.perf_counter() - t3)
    return 0, m


def _block_from_c(b: TjBlock, data: np.ndarray) -> Block:
    """Sub-blocks as column-major views into `data` (no copy)."""
    subs = []
    for i in range(b.num):
        s = b.sub[i]
        n = s.row_dim * s.sdim
        subs.append(SubBlock(s.num_up, s.num_down, s.down_dif,
                             data[s.off:s.off + n].reshape((s.row_dim, s.sdim), order="F")))
    return Block(b.len, b.up_dif, b.down_dif, subs)


class _ResultPack:
    """The packed form of a model the library wrote: its own result arrays."""

    class _P:
        def __init__(self, c, data):
            self.c, self.data = c, data

    def __init__(self, m: TjModel, data: np.ndarray, keep, model: "Model"):
        self.c = m
        self.keep = keep
        self.ham = self._P(m.ham, data)
        self.sets = [[self._P(getattr(m.sub[i], k), data) for k in OPS] for i in range(m.nsub)]
        self.data = data
        self.ham_views = _views(model.ham)
        self.lazy = model.sub

    def matches(self, model: "Model") -> bool:
        if model.sub is not self.lazy or _views(model.ham) != self.ham_views:
            return False
        # only sets that have been built can have been changed: each against
        # the views it was built with
        return all([_views(getattr(bs, k)) for k in OPS] == v for bs, v in self.lazy.built())


class _LazySets(Sequence):
    """Model.sub of a model the library wrote: each BlockSet (its sub-blocks
    views into the result array) is built when first read -- a sweep reads
    only the Hamiltonian of the blocks it passes back."""

    def __init__(self, m: TjModel, data: np.ndarray):
        self._m, self._data = m, data
        self._sets: List[Optional[BlockSet]] = [None] * m.nsub
        self._views: List[Optional[list]] = [None] * m.nsub

    def __len__(self):
        return len(self._sets)

    def __getitem__(self, i):
        if isinstance(i, slice):
            return [self[j] for j in range(*i.indices(len(self)))]
        if i < 0:
            i += len(self)
        if not 0 <= i < len(self):
            raise IndexError(i)
        if self._sets[i] is None:
            bs = self._m.sub[i]
            self._sets[i] = BlockSet(*[_block_from_c(getattr(bs, k), self._data) for k in OPS])
            self._views[i] = [_views(getattr(self._sets[i], k)) for k in OPS]
        return self._sets[i]

    def __eq__(self, other):
        return list(self) == list(other)

    def built(self):
        return [(bs, v) for bs, v in zip(self._sets, self._views) if bs is not None]


def model_from_c(m: TjModel, data: np.ndarray, keep=None) -> Model:
    """A tj_model whose blocks all point into `data` -> a numpy-side Model whose
    sub-blocks are views into `data` (the operator sets built when first
    read); `keep` holds the arrays the C structs point into, so that the Model
    packs without a copy."""
    out = Model(m.len, _block_from_c(m.ham, data), _LazySets(m, data))
    if keep is not None:
        out._packed = _ResultPack(m, data, keep, out)
    return out


def call_block_result(call):
    """Runs a two-call block-result entry point `call(res_ptr) -> rc`; returns (rc, Block)."""
    res = TjBlockResult()
    rc = call(C.byref(res))
    if rc:
        return rc, None
    subs = (TjBlockSub * max(res.num, 1))()
    data = np.zeros(max(res.data_len, 1))
    res.subs = C.cast(subs, C.POINTER(TjBlockSub))
    res.data = data.ctypes.data_as(c_double_p)
    rc = call(C.byref(res))
    if rc:
        return rc, None
    b = _block_from_c(res.block, data)
    b._packed = _BlockView(res.block, subs, data, b)
    return 0, b


class PackedChain:
    """tj_chain of one side's measurement tables: bases[i] / truns[i] for block
    length i (dicts keyed by length, as the sweep driver stores them)."""

    def __init__(self, n: int, bases: dict, truns: dict, trun_idx: int = 1):
        self.bsm = (TjBasis * max(n, 1))()
        self.truns = (TjBlock * max(n, 1))()
        self.keep = []
        for i in range(2, n + 1):
            if i in bases:
                pb = bases[i].pack()
                self.keep.append(pb)
                self.bsm[i - 1] = pb.c
            if i in truns and i > trun_idx:
                pt = truns[i].pack()
                self.keep.append(pt)
                self.truns[i - 1] = pt.c
        self.c = TjChain(n, trun_idx, C.cast(self.bsm, C.POINTER(TjBasis)), C.cast(self.truns, C.POINTER(TjBlock)))


def block_from_c_result(res: TjTruncResult, length: int, subs_arr=None, data: Optional[np.ndarray] = None) -> Block:
    """Turns a filled tj_trunc_result into a Block (trun_op).  Given the
    sub-block table and data array the result was written into, the
    sub-blocks are views into `data` and the Block packs to those arrays
    without a copy; otherwise they are copies."""
    subs = []
    for i in range(res.num):
        s = res.sub[i]
        n = s.row_dim * s.sdim
        if data is not None:
            mat = data[s.off:s.off + n].reshape((s.row_dim, s.sdim), order="F")
        else:
            buf = np.ctypeslib.as_array(res.data, shape=(res.data_len,))[s.off:s.off + n]
            mat = buf.reshape((s.row_dim, s.sdim), order="F").copy()
        subs.append(SubBlock(s.num_up, s.num_down, 0, mat))
    b = Block(length, 0, 0, subs)
    if data is not None and subs_arr is not None:
        b._packed = _BlockView(TjBlock(length, res.num, b.dim, 0, 0, 0, C.cast(subs_arr, C.POINTER(TjBlockSub)),
                                       _dptr(data)), subs_arr, data, b)
    return b
