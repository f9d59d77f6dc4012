"""Python mirror of the reference's routine interface, bound to libtjb200.so.

Each function takes the same objects as the Fortran routine it replaces
(models, bases, wavefunctions) and calls the corresponding C-ABI entry point
of include/tj_b200.h.  There is no CPU path: when the compiled library is
missing or no B200 is visible the calls raise.
"""
from __future__ import annotations

import ctypes as C
import os
import time
import weakref
from typing import Optional, Tuple

import numpy as np

from .structs import (Basis, BasisMap, Block, TjBasis, TjBasisMap, TjBasisResult, TjBasisSub, TjBlock, TjBlockResult, TjBlockSet, TjBlockSub, TjChain, TjGgCell, TjGgTerm,
                      TjHpsiStats, TjLattice, TjModel, TjModelResult, TjTruncResult, TjTuneResult, TjWave, Wave,
                      RESULT_HOST_S, block_from_c_result, call_block_result, call_model_result)

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libtjb200.so")

TJ_PREC_FP64, TJ_PREC_OZAKI = 0, 1
TJ_TUNE_OFF, TJ_TUNE_CACHED, TJ_TUNE_ON_MISS = 0, 1, 2


class TjError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__("tj error %d: %s" % (code, msg))
        self.code = code


class PlanOperand(C.Structure):
    _fields_ = [("off", C.c_int64), ("ld", C.c_int32), ("space", C.c_int8), ("trans", C.c_int8),
                ("pad_", C.c_int16)]


class PlanTask(C.Structure):
    _fields_ = [("L", PlanOperand), ("R", PlanOperand), ("coef", C.c_double), ("K", C.c_int32),
                ("pad_", C.c_int32)]


class PlanCell(C.Structure):
    _fields_ = [("off", C.c_int64), ("ld", C.c_int32), ("M", C.c_int32), ("N", C.c_int32),
                ("t_begin", C.c_int32), ("t_end", C.c_int32), ("space", C.c_int8), ("pad_", C.c_int8 * 7)]


class PlanUpload(C.Structure):
    _fields_ = [("src", C.c_void_p), ("n", C.c_int64), ("dst", C.c_int64)]


class PlanMerge(C.Structure):
    _fields_ = [("dst", C.c_int64), ("n", C.c_int64), ("s_begin", C.c_int32), ("s_end", C.c_int32)]


class PlanItem(C.Structure):
    _fields_ = [(n, C.c_int32) for n in ("cell", "row0", "col0", "tb", "te", "ab", "ae", "slot")]


class PlanReduce(C.Structure):
    _fields_ = [(n, C.c_int32) for n in ("cell", "row0", "col0", "slot0", "nslot", "ab", "ae", "pad_")]


class PlanExport(C.Structure):
    _fields_ = [("ops_len", C.c_int64), ("scratch_len", C.c_int64), ("psi_len", C.c_int64),
                ("n_tasks1", C.c_int64), ("n_tasks2", C.c_int64), ("n_cells1", C.c_int64),
                ("n_cells2", C.c_int64), ("n_uploads", C.c_int64), ("n_merges", C.c_int64),
                ("n_merge_src", C.c_int64), ("flops", C.c_double), ("flops_ref", C.c_double),
                ("bytes", C.c_double),
                ("tasks1", C.POINTER(PlanTask)), ("tasks2", C.POINTER(PlanTask)),
                ("cells1", C.POINTER(PlanCell)), ("cells2", C.POINTER(PlanCell)),
                ("uploads", C.POINTER(PlanUpload)), ("merges", C.POINTER(PlanMerge)),
                ("merge_src", C.POINTER(C.c_int64)), ("merge_coef", C.POINTER(C.c_double)),
                ("n_items1", C.c_int64), ("n_items2", C.c_int64), ("n_red1", C.c_int64), ("n_red2", C.c_int64),
                ("items1", C.POINTER(PlanItem)), ("items2", C.POINTER(PlanItem)),
                ("red1", C.POINTER(PlanReduce)), ("red2", C.POINTER(PlanReduce))]


class OzJobC(C.Structure):
    _fields_ = [("src_off", C.c_int64), ("dst", C.c_int64), ("scale_idx", C.c_int64), ("coef", C.c_double)] + \
               [(n, C.c_int32) for n in ("rs", "ks", "nrows", "K", "gtot", "kb0", "R", "nkb", "ntiles", "gt_last",
                                         "row0")] + \
               [("space", C.c_int8), ("want_max", C.c_int8), ("want_split", C.c_int8), ("pad_", C.c_int8)]


class OzSegC(C.Structure):
    _fields_ = [("a_base", C.c_int64), ("b_base", C.c_int64)] + \
               [(n, C.c_int32) for n in ("a_nkb", "b_nkb", "a_kb0", "b_kb0", "nkb", "pad_")]


class OzFamC(C.Structure):
    _fields_ = [("seg_begin", C.c_int32), ("seg_end", C.c_int32), ("rs_idx", C.c_int64), ("cs_idx", C.c_int64),
                ("nkb", C.c_int32), ("pad_", C.c_int32)]


class OzItemC(C.Structure):
    _fields_ = [(n, C.c_int32) for n in ("kind", "cell", "row0", "col0", "M", "N", "mrows", "ncols", "fam_begin",
                                         "fam_end", "pad1_", "init")] + \
               [("pi_idx", C.c_int64), ("nkb", C.c_int32), ("pad2_", C.c_int32), ("cost", C.c_int64)]


class OzCellC(C.Structure):
    _fields_ = [("off", C.c_int64)] + [(n, C.c_int32) for n in ("ld", "M", "N", "a_begin", "a_end", "pad_")]


class OzProwC(C.Structure):
    _fields_ = [(n, C.c_int32) for n in ("row_begin", "rows", "ld", "pad_")] + [("off", C.c_int64), ("pi", C.c_int64)]


_OZ_ARRAYS = [("sta_jobs", OzJobC), ("psi_jobs", OzJobC), ("prod_jobs", OzJobC), ("segs", OzSegC),
              ("fams", OzFamC), ("cells", OzCellC), ("items1", OzItemC), ("items2", OzItemC)]


class OzExport(C.Structure):
    _fields_ = ([("slices", C.c_int32), ("tile_n", C.c_int32)] +
                [(n, C.c_int64) for n in ("sta_pack", "dyn_pack", "n_scales", "rho0", "tau0", "pi0")] +
                [("int8_ops", C.c_double)] +
                [("n_" + n, C.c_int64) for n, _ in _OZ_ARRAYS] +
                [(n, C.POINTER(t)) for n, t in _OZ_ARRAYS] +
                [("n_cta1", C.c_int64), ("n_cta2", C.c_int64), ("cta1", C.POINTER(C.c_int32)),
                 ("cta2", C.POINTER(C.c_int32)), ("n_sta_mjobs", C.c_int64), ("n_psi_mjobs", C.c_int64),
                 ("n_prod_mjobs", C.c_int64), ("sta_mjobs", C.POINTER(OzJobC)), ("psi_mjobs", C.POINTER(OzJobC)),
                 ("prod_mjobs", C.POINTER(OzJobC)), ("n_prod_rows", C.c_int64), ("prod_rows", C.POINTER(OzProwC))])


_lib = None


class _Lib:
    """Wraps the CDLL; argtypes of symbols the library does not export are skipped."""

    def __init__(self, dll):
        object.__setattr__(self, "_dll", dll)

    def __getattr__(self, name):
        try:
            return getattr(self._dll, name)
        except AttributeError:
            return _Missing(name)


class _Missing:
    def __init__(self, name):
        self.name = name

    def __setattr__(self, k, v):
        object.__setattr__(self, k, v)

    def __call__(self, *a):
        raise TjError(-1, "libtjb200.so does not export " + self.name)


COR_NAMES = {
    "measure_sys_block": 0, "measure_env_block": 1, "sys_block_env_block_cor_dia": 2,
    "sys_block_env_block_cor_ndia": 3, "sys_block_site_cor_ndia": 4, "env_block_site_cor_ndia": 5,
    "sys_block_env_site_cor_ndia": 6, "sys_site_env_block_cor_ndia": 7, "sys_site_env_site_cor_ndia": 8,
}


def lib():
    """Loads libtjb200.so (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise OSError("libtjb200.so not built: run python -m grand_sql_tj_b200.build")
        L = _Lib(C.CDLL(LIB_PATH))
        P = C.POINTER
        L.tj_last_error.restype = C.c_char_p
        L.tj_ctx_create.argtypes = [P(C.c_void_p), C.c_int]
        L.tj_ctx_destroy.argtypes = [C.c_void_p]
        L.tj_set_precision.argtypes = [C.c_void_p, C.c_int, C.c_int]
        L.tj_step_begin.argtypes = [C.c_void_p]
        L.tj_set_wait_limit.argtypes = [C.c_void_p, C.c_double]
        L.tj_set_residency.argtypes = [C.c_void_p, C.c_double]
        L.tj_residency_forget.argtypes = [C.c_void_p, C.c_void_p]
        L.tj_host_register.argtypes = [C.c_void_p, C.c_size_t]
        L.tj_host_unregister.argtypes = [C.c_void_p]
        hp = [C.c_void_p, P(TjLattice), P(TjModel), P(TjModel), P(TjBasis), P(TjBasis)]
        L.tj_model_wave.argtypes = hp + [P(TjWave), P(TjWave)]
        L.tj_model_wave_bench.argtypes = hp + [P(TjWave), P(TjWave), C.c_int, P(C.c_double)]
        L.tj_lanczos_memo_new.argtypes = hp + [P(TjWave), C.c_int, C.c_double, P(C.c_double), P(C.c_int)]
        L.tj_truncation.argtypes = [C.c_void_p, P(TjWave), C.c_int, C.c_int, C.c_int, C.c_double,
                                    P(TjTruncResult)]
        L.tj_hpsi_stats_get.argtypes = [C.c_void_p, P(TjHpsiStats)]
        L.tj_set_autotune.argtypes = [C.c_void_p, C.c_int]
        L.tj_model_wave_multi.argtypes = [C.c_void_p, C.c_int, P(P(TjLattice)), P(P(TjModel)), P(P(TjModel)),
                                          P(P(TjBasis)), P(P(TjBasis)), P(P(TjWave)), P(P(TjWave)), C.c_int,
                                          P(C.c_double)]
        L.tj_autotune.argtypes = [C.c_void_p, P(TjLattice), P(TjModel), P(TjModel), P(TjBasis), P(TjBasis),
                                  P(TjWave), P(TjTuneResult)]
        L.tj_grouped_gemm_bench.argtypes = [C.c_void_p, P(TjGgCell), C.c_int, P(TjGgTerm), C.c_int,
                                            P(C.c_double), C.c_int64, C.c_int64, C.c_int, C.c_int,
                                            P(C.c_double), P(C.c_double), P(C.c_double), P(TjTuneResult)]
        L.tj_hpsi_plan_export.argtypes = [P(TjLattice), P(TjModel), P(TjModel), P(TjBasis), P(TjBasis),
                                          P(TjWave), P(PlanExport)]
        L.tj_cor_plan_export.argtypes = [C.c_int, P(TjBlock), P(TjBlock), P(TjBasis), P(TjBasis), P(TjWave),
                                         C.c_char, P(PlanExport)]
        L.tj_ozaki_plan_export.argtypes = [P(TjLattice), P(TjModel), P(TjModel), P(TjBasis), P(TjBasis),
                                           P(TjWave), C.c_int, P(OzExport)]
        L.tj_get_hamiltonian.argtypes = [C.c_void_p, P(TjLattice), C.c_int, C.c_int, P(TjModel), P(TjBasis),
                                         P(TjBlock), P(TjModelResult)]
        L.tj_renorm_plan_export.argtypes = [P(TjLattice), C.c_int, C.c_int, P(TjModel), P(TjBasis), P(TjBlock),
                                            P(PlanExport), P(TjModelResult)]
        L.tj_wave_trans.argtypes = [C.c_void_p, C.c_int, P(TjBasis), P(TjBasis), P(TjBlock), P(TjBlock), P(TjWave),
                                    P(TjWave)]
        L.tj_wave_trans_plan_export.argtypes = [C.c_int, P(TjBasis), P(TjBasis), P(TjBlock), P(TjBlock), P(TjWave),
                                                P(TjWave), P(PlanExport)]
        L.tj_get_oper.argtypes = [C.c_void_p, C.c_int, C.c_int, P(TjChain), P(TjBlock), C.c_int, C.c_int, C.c_int,
                                  C.c_char, P(TjBlockResult)]
        L.tj_change_oper.argtypes = L.tj_get_oper.argtypes
        L.tj_update_trun.argtypes = [C.c_void_p, C.c_int, P(TjBlock), P(TjBlock), P(TjBlockResult)]
        L.tj_block_mul_block_ndia.argtypes = [C.c_void_p, P(TjBlock), C.c_char, P(TjBlock), C.c_char, C.c_double,
                                              C.c_int, P(TjBasis), P(TjBlockResult)]
        L.tj_disk_name.argtypes = [C.c_int, C.c_int, C.c_char_p, C.c_int]
        L.tj_wave_to_disk.argtypes = [C.c_char_p, P(TjWave)]
        L.tj_wave_from_disk.argtypes = [C.c_char_p, P(TjWave), C.c_void_p, C.c_void_p]
        L.tj_block_to_disk.argtypes = [C.c_char_p, P(TjBlock)]
        L.tj_block_from_disk.argtypes = [C.c_char_p, P(TjBlockResult)]
        L.tj_model_to_disk.argtypes = [C.c_char_p, P(TjModel)]
        L.tj_model_from_disk.argtypes = [C.c_char_p, P(TjModelResult)]
        L.tj_basis_to_disk.argtypes = [C.c_char_p, P(TjBasis)]
        L.tj_basis_from_disk.argtypes = [C.c_char_p, P(TjBasisResult)]
        L.tj_w6js.restype = C.c_double
        L.tj_w6js.argtypes = [C.c_int] * 6
        L.tj_w3js.restype = C.c_double
        L.tj_w3js.argtypes = [C.c_int] * 6
        for n in ("tj_measure_sys_block", "tj_measure_env_block"):
            getattr(L, n).argtypes = [C.c_void_p, P(TjBlock), P(TjBasis), P(TjWave), P(C.c_double)]
        L.tj_sys_block_env_block_cor_dia.argtypes = [C.c_void_p, P(TjBlock), P(TjBlock), P(TjBasis),
                                                     P(TjBasis), P(TjWave), P(C.c_double)]
        for n in ("tj_sys_block_env_block_cor_ndia", "tj_sys_block_env_site_cor_ndia",
                  "tj_sys_site_env_block_cor_ndia", "tj_sys_site_env_site_cor_ndia"):
            getattr(L, n).argtypes = [C.c_void_p, P(TjBlock), P(TjBlock), P(TjBasis), P(TjBasis),
                                      P(TjWave), C.c_char, P(C.c_double)]
        for n in ("tj_sys_block_site_cor_ndia", "tj_env_block_site_cor_ndia"):
            getattr(L, n).argtypes = [C.c_void_p, P(TjBlock), P(TjBlock), P(TjBasis), P(TjWave),
                                      C.c_char, P(C.c_double)]
        _lib = L
    return _lib


def _chk(rc: int):
    if rc:
        raise TjError(rc, lib().tj_last_error().decode())


class _PoolView:
    """The owner of the numpy arrays made from one pool buffer: every view and
    every slice of them refers to it, so it dies only with the last of them."""

    def __init__(self, ptr: int, n: int):
        self.__array_interface__ = {"shape": (n,), "typestr": "<f8", "data": (ptr, False), "version": 3}


class HostPool:
    """Page-locked host buffers reused for arrays the library writes (blocks,
    wavefunctions).  Each buffer is registered once (tj_host_register), so
    the device writes it by DMA at full rate, and goes back to the pool when
    the last array (or slice) made from it is freed, so that its pages are not
    faulted in and pinned again for the next array.  Sizes are rounded up to
    eight classes per octave."""

    def __init__(self):
        self.free = {}
        self.bufs = []   # every buffer (kept alive here for the process)

    @staticmethod
    def size_class(n: int) -> int:
        if n <= 1 << 12:
            return 1 << 12
        q = 1 << (n.bit_length() - 4)
        return (n + q - 1) // q * q

    def get(self, n: int) -> np.ndarray:
        c = self.size_class(n)
        lst = self.free.get(c)
        if lst:
            buf = lst.pop()
        else:
            buf = (C.c_double * c)()
            _chk(lib().tj_host_register(C.addressof(buf), C.sizeof(buf)))
            self.bufs.append(buf)
        owner = _PoolView(C.addressof(buf), n)
        weakref.finalize(owner, self._put, c, buf)
        return np.asarray(owner)

    def _put(self, c: int, buf):
        self.free.setdefault(c, []).append(buf)

    def reserve(self, sizes):
        """Registers buffers for arrays of the given sizes ahead of use (the
        registration, not the later use, then carries the pinning cost)."""
        held = [self.get(n) for n in sizes]
        del held


# One pool per process: page-locked memory serves every context of the device.
HOST_POOL = HostPool()


class Context:
    """One tj_ctx: a CUDA device, a stream and the cached plan of the current step."""

    def __init__(self, device: int = 0):
        self.h = C.c_void_p()
        self.resident = False
        self.pool: Optional[HostPool] = None
        _chk(lib().tj_ctx_create(C.byref(self.h), device))

    def use_host_pool(self, on: bool = True):
        """Blocks from get_hamiltonian and the sweep's wavefunctions go into
        page-locked, reused host buffers (the process's HostPool)."""
        self.pool = HOST_POOL if on else None

    def set_residency(self, gigabytes: float):
        """tj_set_residency: keep the blocks get_hamiltonian returns on the device
        (budget in GB; 0 turns it off).  Each returned Model's array is dropped
        from the device when the Model is freed."""
        _chk(lib().tj_set_residency(self.h, float(gigabytes)))
        self.resident = gigabytes > 0

    def _forget_when_freed(self, arr: np.ndarray):
        ref = weakref.ref(self)
        ptr = arr.ctypes.data

        def forget():
            c = ref()
            if c is not None and c.h:
                lib().tj_residency_forget(c.h, C.c_void_p(ptr))
        weakref.finalize(arr, forget)

    def close(self):
        if self.h:
            lib().tj_ctx_destroy(self.h)
            self.h = C.c_void_p()
        self.pool = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_precision(self, mode: int, slices: int = 6):
        _chk(lib().tj_set_precision(self.h, mode, slices))

    def step_begin(self):
        _chk(lib().tj_step_begin(self.h))

    def set_wait_limit(self, seconds: float):
        _chk(lib().tj_set_wait_limit(self.h, seconds))

    def stats(self) -> TjHpsiStats:
        s = TjHpsiStats()
        _chk(lib().tj_hpsi_stats_get(self.h, C.byref(s)))
        return s

    def model_wave_multi(self, sbs, reps: int = 0, invecs=None):
        """tj_model_wave_multi: H*psi of independent superblocks in shared launches.
        Returns (outputs, ms of one shared product when reps > 0)."""
        P = C.POINTER
        n = len(sbs)
        invecs = [sb.wave for sb in sbs] if invecs is None else invecs
        packs = [pack_superblock(sb) for sb in sbs]
        outs = [w.like() for w in invecs]
        arr = lambda t, xs: (P(t) * n)(*[C.pointer(x) for x in xs])
        lat = arr(TjLattice, [sb.lat.c for sb in sbs])
        sysm = arr(TjModel, [p[0].c for p in packs])
        envm = arr(TjModel, [p[1].c for p in packs])
        sbs_ = arr(TjBasis, [p[2].c for p in packs])
        ebs_ = arr(TjBasis, [p[3].c for p in packs])
        ins = arr(TjWave, [w.c for w in invecs])
        ous = arr(TjWave, [w.c for w in outs])
        ms = C.c_double()
        _chk(lib().tj_model_wave_multi(self.h, n, lat, sysm, envm, sbs_, ebs_, ins, ous, reps, C.byref(ms)))
        return outs, (ms.value if reps > 0 else None)

    def set_autotune(self, mode: int):
        _chk(lib().tj_set_autotune(self.h, mode))

    def autotune(self, sb, packed=None) -> TjTuneResult:
        """tj_autotune: searches the tiling choices for this superblock's block-size histogram."""
        ps, pe, bs, be = packed if packed is not None else pack_superblock(sb)
        r = TjTuneResult()
        _chk(lib().tj_autotune(self.h, C.byref(sb.lat.c), C.byref(ps.c), C.byref(pe.c), C.byref(bs.c),
                               C.byref(be.c), C.byref(sb.wave.c), C.byref(r)))
        return r

    def grouped_gemm_bench(self, batch, mode: int, reps: int = 3):
        """tj_grouped_gemm_bench on a GgBatch: (ms per repetition, output, flops, tune result or None)."""
        out = np.zeros(batch.out_len)
        ms, fl = C.c_double(), C.c_double()
        tr = TjTuneResult()
        _chk(lib().tj_grouped_gemm_bench(self.h, batch.cells, len(batch.cells), batch.terms, len(batch.terms),
                                         batch.pool.ctypes.data_as(C.POINTER(C.c_double)), batch.pool.size,
                                         batch.out_len, mode, reps, out.ctypes.data_as(C.POINTER(C.c_double)),
                                         C.byref(ms), C.byref(fl), C.byref(tr)))
        return ms.value, out, fl.value, (tr if mode == 2 else None)

    # --------------------------------------------------------- hot path
    def model_wave(self, sb, invec: Optional[Wave] = None) -> Wave:
        """model_wave (get_sys.f90:4127) with hmerge; host buffers in and out."""
        invec = sb.wave if invec is None else invec
        ps, pe, bs, be = sb.sys.pack(), sb.env.pack(), sb.sys_bs.pack(), sb.env_bs.pack()
        out = invec.like()
        _chk(lib().tj_model_wave(self.h, C.byref(sb.lat.c), C.byref(ps.c), C.byref(pe.c), C.byref(bs.c),
                                 C.byref(be.c), C.byref(invec.c), C.byref(out.c)))
        return out

    def model_wave_bench(self, sb, reps: int, invec: Optional[Wave] = None) -> Tuple[float, Wave]:
        invec = sb.wave if invec is None else invec
        ps, pe, bs, be = sb.sys.pack(), sb.env.pack(), sb.sys_bs.pack(), sb.env_bs.pack()
        out = invec.like()
        ms = C.c_double()
        _chk(lib().tj_model_wave_bench(self.h, C.byref(sb.lat.c), C.byref(ps.c), C.byref(pe.c), C.byref(bs.c),
                                       C.byref(be.c), C.byref(invec.c), C.byref(out.c), reps, C.byref(ms)))
        return ms.value, out

    def lanczos_memo_new(self, sb, lanzero: float, start: Optional[Wave] = None, packed=None,
                         in_place: bool = False):
        """lanczos_memo_new (eigen.f90:2), levels = 1: returns (E0, iterations, Ritz vector).

        packed: (sys, env, sys_bs, env_bs) from pack_superblock, reused across
        calls; in_place: `start` is overwritten by the Ritz vector (as the
        reference's eigvec argument is) instead of being copied first."""
        w = sb.wave if start is None else start
        if not in_place:
            w = w.copy()
        ps, pe, bs, be = packed if packed is not None else pack_superblock(sb)
        e, it = (C.c_double * 1)(), C.c_int()
        _chk(lib().tj_lanczos_memo_new(self.h, C.byref(sb.lat.c), C.byref(ps.c), C.byref(pe.c), C.byref(bs.c),
                                       C.byref(be.c), C.byref(w.c), 1, lanzero, e, C.byref(it)))
        if self.resident:
            self._forget_when_freed(w.data)
        return e[0], it.value, w

    def lanczos(self, lat, sys, env, sys_bs, env_bs, wave: Wave, lanzero: float, in_place: bool = False):
        """lanczos_memo_new on explicit models and bases: returns (E0, iterations, Ritz vector);
        in_place: the Ritz vector overwrites `wave` (else a copy)."""
        w = wave if in_place else wave.copy()
        ps, pe, bs, be = sys.pack(), env.pack(), sys_bs.pack(), env_bs.pack()
        e, it = (C.c_double * 1)(), C.c_int()
        _chk(lib().tj_lanczos_memo_new(self.h, C.byref(lat.c), C.byref(ps.c), C.byref(pe.c), C.byref(bs.c),
                                       C.byref(be.c), C.byref(w.c), 1, lanzero, e, C.byref(it)))
        return e[0], it.value, w

    def get_hamiltonian(self, lat, side: int, mshift: int, pre, basis, trun: Block):
        """Get_Hamiltonian_Sys (side 0) / Get_Hamiltonian_Env (side 1) (get_sys.f90:4-480):
        the Model `pre` enlarged into `basis` and truncated with `trun`; returns the new Model."""
        pp, pb, pt = pre.pack(), basis.pack(), trun.pack()
        rc, m = call_model_result(lambda r: lib().tj_get_hamiltonian(self.h, C.byref(lat.c), side, mshift,
                                                                     C.byref(pp.c), C.byref(pb.c), C.byref(pt.c), r),
                                  alloc=self.pool.get if self.pool is not None else None)
        _chk(rc)
        if self.resident:
            self._forget_when_freed(m._packed.data)
        return m

    def wave_trans(self, direction: int, sys_bs, env_bs, sys_trun: Block, env_trun: Block, old: Wave,
                   new_wave: Wave) -> Wave:
        """wave_trans_LR (direction 0) / wave_trans_RL (direction 1) (dmrg_sub.f90:1093-1384):
        fills `new_wave` (the next superblock's sectors) and returns it."""
        pb, pe, ps, pt = sys_bs.pack(), env_bs.pack(), sys_trun.pack(), env_trun.pack()
        _chk(lib().tj_wave_trans(self.h, direction, C.byref(pb.c), C.byref(pe.c), C.byref(ps.c), C.byref(pt.c),
                                 C.byref(old.c), C.byref(new_wave.c)))
        if self.resident:
            self._forget_when_freed(new_wave.data)
        return new_wave

    def get_oper(self, side: int, dia: int, chain, st_oper: Block, old_idx: int, new_idx: int, truns: bool,
                 types: str = "B") -> Block:
        """Get_{sys,env}_oper_{dia,ndia} (get_sys.f90:764-1130); chain: structs.PackedChain."""
        ps = st_oper.pack()
        rc, b = call_block_result(lambda r: lib().tj_get_oper(self.h, side, int(dia), C.byref(chain.c), C.byref(ps.c),
                                                              old_idx, new_idx, int(truns), types.encode(), r))
        _chk(rc)
        return b

    def change_oper(self, side: int, dia: int, chain, old_oper: Block, old_idx: int, new_idx: int, truns: bool,
                    types: str = "B") -> Block:
        """Change_{sys,env}_oper_{dia,ndia} (get_sys.f90:893-1238)."""
        ps = old_oper.pack()
        rc, b = call_block_result(lambda r: lib().tj_change_oper(self.h, side, int(dia), C.byref(chain.c),
                                                                 C.byref(ps.c), old_idx, new_idx, int(truns),
                                                                 types.encode(), r))
        _chk(rc)
        return b

    def update_trun(self, dia: int, ori: Block, trun: Block) -> Block:
        """update_trun_dia / update_trun_ndia (block.f90:1311-1503)."""
        po, pt = ori.pack(), trun.pack()
        rc, b = call_block_result(lambda r: lib().tj_update_trun(self.h, int(dia), C.byref(po.c), C.byref(pt.c), r))
        _chk(rc)
        return b

    def block_mul_block_ndia(self, o1: Block, f1: str, o2: Block, f2: str, coef: float, down_dif: int, basis) -> Block:
        """block_mul_block_ndia (block.f90:1956-2197)."""
        p1, p2, pb = o1.pack(), o2.pack(), basis.pack()
        rc, b = call_block_result(lambda r: lib().tj_block_mul_block_ndia(self.h, C.byref(p1.c), f1.encode(),
                                                                          C.byref(p2.c), f2.encode(), coef, down_dif,
                                                                          C.byref(pb.c), r))
        _chk(rc)
        return b

    def truncation(self, wave: Wave, side: int, kept_min: int, kept_max: int, trun_err: float):
        """Get_density_matrix_{sys,env}_new + Get_truncation_operator (den_mat.f90)."""
        r = TjTruncResult()
        _chk(lib().tj_truncation(self.h, C.byref(wave.c), side, kept_min, kept_max, trun_err, C.byref(r)))
        subs = (TjBlockSub * max(r.num, 1))()
        # the library writes every entry: a pooled page-locked buffer takes the copy at the DMA rate
        data = self.pool.get(max(r.data_len, 1)) if self.pool is not None else np.zeros(max(r.data_len, 1))
        r.sub = C.cast(subs, C.POINTER(TjBlockSub))
        r.data = data.ctypes.data_as(C.POINTER(C.c_double))
        _chk(lib().tj_truncation(self.h, C.byref(wave.c), side, kept_min, kept_max, trun_err, C.byref(r)))
        if self.resident:
            self._forget_when_freed(data)
        length = wave.sys_len if side == 0 else wave.env_len
        return r, block_from_c_result(r, length, subs, data)

    def correlator(self, name: str, a: Block, b: Optional[Block], sys_bs, env_bs, wave: Wave,
                   flag: str = "B") -> float:
        """The measure.f90 contraction `name` (e.g. 'sys_block_env_block_cor_ndia')."""
        L = lib()
        v = C.c_double()
        pa = a.pack()
        pb = b.pack() if b is not None else None
        ps = sys_bs.pack() if sys_bs is not None else None
        pe = env_bs.pack() if env_bs is not None else None
        fn = getattr(L, "tj_" + name)
        f = flag.encode()
        if name == "measure_sys_block":
            _chk(fn(self.h, C.byref(pa.c), C.byref(ps.c), C.byref(wave.c), C.byref(v)))
        elif name == "measure_env_block":
            _chk(fn(self.h, C.byref(pa.c), C.byref(pe.c), C.byref(wave.c), C.byref(v)))
        elif name == "sys_block_env_block_cor_dia":
            _chk(fn(self.h, C.byref(pa.c), C.byref(pb.c), C.byref(ps.c), C.byref(pe.c), C.byref(wave.c),
                    C.byref(v)))
        elif name == "sys_block_site_cor_ndia":
            _chk(fn(self.h, C.byref(pa.c), C.byref(pb.c), C.byref(ps.c), C.byref(wave.c), f, C.byref(v)))
        elif name == "env_block_site_cor_ndia":
            _chk(fn(self.h, C.byref(pa.c), C.byref(pb.c), C.byref(pe.c), C.byref(wave.c), f, C.byref(v)))
        else:
            _chk(fn(self.h, C.byref(pa.c), C.byref(pb.c), C.byref(ps.c), C.byref(pe.c), C.byref(wave.c), f,
                    C.byref(v)))
        return v.value


def _export(call) -> dict:
    ex = PlanExport()
    _chk(call(C.byref(ex)))
    arrs = {
        "tasks1": (PlanTask * max(ex.n_tasks1, 1))(), "tasks2": (PlanTask * max(ex.n_tasks2, 1))(),
        "cells1": (PlanCell * max(ex.n_cells1, 1))(), "cells2": (PlanCell * max(ex.n_cells2, 1))(),
        "uploads": (PlanUpload * max(ex.n_uploads, 1))(), "merges": (PlanMerge * max(ex.n_merges, 1))(),
        "merge_src": (C.c_int64 * max(ex.n_merge_src, 1))(), "merge_coef": (C.c_double * max(ex.n_merge_src, 1))(),
        "items1": (PlanItem * max(ex.n_items1, 1))(), "items2": (PlanItem * max(ex.n_items2, 1))(),
        "red1": (PlanReduce * max(ex.n_red1, 1))(), "red2": (PlanReduce * max(ex.n_red2, 1))(),
    }
    for k, a in arrs.items():
        setattr(ex, k, C.cast(a, type(getattr(ex, k))))
    _chk(call(C.byref(ex)))
    # copy the operator data now, while the caller's packed buffers are alive
    ops = np.zeros(max(ex.ops_len, 1))
    for i in range(ex.n_uploads):
        u = arrs["uploads"][i]
        src = np.ctypeslib.as_array(C.cast(u.src, C.POINTER(C.c_double)), shape=(u.n,))
        ops[u.dst:u.dst + u.n] = src
    return {"ex": ex, "ops": ops, **arrs}


def renorm_plan_export(lat, side: int, mshift: int, pre, basis, trun: Block) -> dict:
    """Compiled task lists of tj_get_hamiltonian (no GPU needed), with the
    result's records: {"ex", "ops", ..., "trun": trun data, "res": TjModelResult}."""
    L = lib()
    pp, pb, pt = pre.pack(), basis.pack(), trun.pack()
    res = TjModelResult()
    _chk(L.tj_renorm_plan_export(C.byref(lat.c), side, mshift, C.byref(pp.c), C.byref(pb.c), C.byref(pt.c),
                                 C.byref(PlanExport()), C.byref(res)))
    sets = (TjBlockSet * max(res.nsub, 1))()
    subs = (TjBlockSub * max(res.n_subs, 1))()
    dummy = np.zeros(1)
    res.sets = C.cast(sets, C.POINTER(TjBlockSet))
    res.subs = C.cast(subs, C.POINTER(TjBlockSub))
    res.data = dummy.ctypes.data_as(C.POINTER(C.c_double))
    d = _export(lambda ex: L.tj_renorm_plan_export(C.byref(lat.c), side, mshift, C.byref(pp.c), C.byref(pb.c),
                                                    C.byref(pt.c), ex, C.byref(res)))
    lo = min((pt.subs[i].off for i in range(len(trun.subs))), default=0)
    d.update(trun=pt.data[lo:].copy(), res=res, res_arrays=(sets, subs, dummy))
    return d


def wave_trans_plan_export(direction: int, sys_bs, env_bs, sys_trun: Block, env_trun: Block, old: Wave,
                           new_wave: Wave) -> dict:
    """Compiled task lists of tj_wave_trans (no GPU needed)."""
    L = lib()
    pb, pe, ps, pt = sys_bs.pack(), env_bs.pack(), sys_trun.pack(), env_trun.pack()
    return _export(lambda ex: L.tj_wave_trans_plan_export(direction, C.byref(pb.c), C.byref(pe.c), C.byref(ps.c),
                                                           C.byref(pt.c), C.byref(old.c), C.byref(new_wave.c), ex))


class DeviceBackend:
    """The hot-path calls of grand_sql_tj_b200.sweep.Dmrg on the B200, through the C ABI."""

    def __init__(self, ctx: Context, trace: Optional[list] = None):
        self.ctx = ctx
        self.trace = trace   # if a list: (call, the context's statistics after it) per step call

    def _traced(self, name, fn):
        """Runs fn(); with a trace, records (call, the context's statistics
        after it, its wall time in s, host stage times of a model result)."""
        if self.trace is None:
            return fn()
        t0 = time.perf_counter()
        r = fn()
        wall = time.perf_counter() - t0
        self.trace.append((name, self.ctx.stats(), wall,
                           dict(RESULT_HOST_S) if name == "get_hamiltonian" else None))
        return r

    def lanczos(self, lat, sys, env, sys_bs, env_bs, wave, lanzero):
        # the sweep does not reuse its start vector: the Ritz vector overwrites it
        return self._traced("lanczos", lambda: self.ctx.lanczos(lat, sys, env, sys_bs, env_bs, wave, lanzero,
                                                                in_place=True))

    def truncation(self, wave, side, kept_min, kept_max, trun_err):
        return self._traced("truncation", lambda: self.ctx.truncation(wave, side, kept_min, kept_max, trun_err))

    def get_hamiltonian(self, lat, side, mshift, pre, basis, trun):
        return self._traced("get_hamiltonian", lambda: self.ctx.get_hamiltonian(lat, side, mshift, pre, basis, trun))

    def wave_trans(self, direction, sys_bs, env_bs, sys_trun, env_trun, old, new_wave):
        if self.ctx.pool is not None:   # the predicted vector goes into a pooled page-locked buffer
            new_wave = Wave(new_wave.sys_len, new_wave.env_len, new_wave.sectors,
                            self.ctx.pool.get(max(new_wave.dim, 1)))
        return self._traced("wave_trans", lambda: self.ctx.wave_trans(direction, sys_bs, env_bs, sys_trun, env_trun,
                                                                      old, new_wave))

    def get_oper(self, side, dia, chain, st_oper, old_idx, new_idx, truns, types="B"):
        return self.ctx.get_oper(side, dia, chain, st_oper, old_idx, new_idx, truns, types)

    def change_oper(self, side, dia, chain, old_oper, old_idx, new_idx, truns, types="B"):
        return self.ctx.change_oper(side, dia, chain, old_oper, old_idx, new_idx, truns, types)

    def update_trun(self, dia, ori, trun):
        return self.ctx.update_trun(dia, ori, trun)

    def block_mul_block_ndia(self, o1, f1, o2, f2, coef, down_dif, basis):
        return self.ctx.block_mul_block_ndia(o1, f1, o2, f2, coef, down_dif, basis)

    def correlator(self, name, a, b, sys_bs, env_bs, wave, flag="B"):
        return self.ctx.correlator(name, a, b, sys_bs, env_bs, wave, flag)


# ------------------------------------------------------------ checkpoint files
def disk_name(kind: int, idx: int) -> str:
    """The reference's file name: kind 0 sysblocks, 1 systruns, 2 sysbs, 3 envblocks, 4 envtruns, 5 envbs, 6 eigvec."""
    buf = C.create_string_buffer(64)
    _chk(lib().tj_disk_name(kind, idx, buf, 64))
    return buf.value.decode()


def wave_to_disk(path: str, wave: Wave):
    _chk(lib().tj_wave_to_disk(path.encode(), C.byref(wave.c)))


def wave_from_disk(path: str) -> Wave:
    from .structs import TjWaveSub, WaveSector
    L = lib()
    hdr = TjWave()
    _chk(L.tj_wave_from_disk(path.encode(), C.byref(hdr), None, None))
    subs = (TjWaveSub * max(hdr.num, 1))()
    data = np.zeros(max(hdr.dim, 1))
    _chk(L.tj_wave_from_disk(path.encode(), C.byref(hdr), C.cast(subs, C.c_void_p), data.ctypes.data))
    secs = [WaveSector(s.sys_num_up, s.sys_num_down, s.env_num_up, s.env_num_down, s.sys_dim, s.env_dim)
            for s in subs[:hdr.num]]
    return Wave(hdr.sys_len, hdr.env_len, secs, data)


def block_to_disk(path: str, block: Block):
    pb = block.pack()
    _chk(lib().tj_block_to_disk(path.encode(), C.byref(pb.c)))


def block_from_disk(path: str) -> Block:
    rc, b = call_block_result(lambda r: lib().tj_block_from_disk(path.encode(), r))
    _chk(rc)
    return b


def model_to_disk(path: str, model):
    pm = model.pack()
    _chk(lib().tj_model_to_disk(path.encode(), C.byref(pm.c)))


def model_from_disk(path: str):
    rc, m = call_model_result(lambda r: lib().tj_model_from_disk(path.encode(), r))
    _chk(rc)
    return m


def basis_to_disk(path: str, basis: Basis):
    pb = basis.pack()
    _chk(lib().tj_basis_to_disk(path.encode(), C.byref(pb.c)))


def basis_from_disk(path: str) -> Basis:
    L = lib()
    r = TjBasisResult()
    _chk(L.tj_basis_from_disk(path.encode(), C.byref(r)))
    sub = (TjBasisMap * max(r.num, 1))()
    maps = (TjBasisSub * max(r.nmaps, 1))()
    r.sub = C.cast(sub, C.POINTER(TjBasisMap))
    r.maps = C.cast(maps, C.POINTER(TjBasisSub))
    _chk(L.tj_basis_from_disk(path.encode(), C.byref(r)))
    out = []
    for i in range(r.num):
        m = sub[i]
        out.append(BasisMap(m.new_num_up, m.new_num_down,
                            [(q.spos, q.sdim, q.bl_num_up, q.bl_num_down, q.st_num_up, q.st_num_down)
                             for q in maps[m.first:m.first + m.num]]))
    return Basis(r.len, out)


def pack_superblock(sb):
    """The C views (sys, env, sys_bs, env_bs) of a superblock's models and bases."""
    return sb.sys.pack(), sb.env.pack(), sb.sys_bs.pack(), sb.env_bs.pack()


def packed_arrays(packed):
    """Every operator data array of pack_superblock's models (each array once)."""
    out, seen = [], set()
    for m in packed[:2]:
        for a in [m.ham.data] + [p.data for sets in m.sets for p in sets]:
            if id(a) not in seen:
                seen.add(id(a))
                out.append(a)
    return out


class PinnedHost:
    """Page-locks host arrays through tj_host_register for the life of the object."""

    def __init__(self, arrays):
        self.ptrs = []
        for a in arrays:
            if a.nbytes:
                _chk(lib().tj_host_register(a.ctypes.data, a.nbytes))
                self.ptrs.append(a.ctypes.data)

    def close(self):
        for p in self.ptrs:
            lib().tj_host_unregister(p)
        self.ptrs = []

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()


def plan_export(sb, invec: Optional[Wave] = None) -> dict:
    """Compiled task lists of H*psi for `sb` (no GPU needed)."""
    L = lib()
    invec = sb.wave if invec is None else invec
    ps, pe, bs, be = sb.sys.pack(), sb.env.pack(), sb.sys_bs.pack(), sb.env_bs.pack()
    return _export(lambda ex: L.tj_hpsi_plan_export(C.byref(sb.lat.c), C.byref(ps.c), C.byref(pe.c), C.byref(bs.c),
                                                     C.byref(be.c), C.byref(invec.c), ex))


def cor_plan_export(name: str, a: Block, b: Optional[Block], sys_bs, env_bs, wave: Wave, flag: str = "B") -> dict:
    """Compiled task lists of the correlator contraction `name` (no GPU needed)."""
    L = lib()
    pa = a.pack()
    pb = b.pack() if b is not None else None
    ps = sys_bs.pack() if sys_bs is not None else None
    pe = env_bs.pack() if env_bs is not None else None
    ref = lambda p: C.byref(p.c) if p is not None else None
    return _export(lambda ex: L.tj_cor_plan_export(COR_NAMES[name], ref(pa), ref(pb), ref(ps), ref(pe),
                                                    C.byref(wave.c), flag.encode(), ex))


def ozaki_plan_export(sb, slices: int = 5, invec: Optional[Wave] = None) -> dict:
    """Split-precision tables of H*psi for `sb` (no GPU needed)."""
    L = lib()
    invec = sb.wave if invec is None else invec
    ps, pe, bs, be = sb.sys.pack(), sb.env.pack(), sb.sys_bs.pack(), sb.env_bs.pack()

    def call(ex):
        return L.tj_ozaki_plan_export(C.byref(sb.lat.c), C.byref(ps.c), C.byref(pe.c), C.byref(bs.c),
                                      C.byref(be.c), C.byref(invec.c), slices, ex)

    ex = OzExport()
    _chk(call(C.byref(ex)))
    arrs = {n: (t * max(getattr(ex, "n_" + n), 1))() for n, t in _OZ_ARRAYS}
    arrs["cta1"] = (C.c_int32 * max(ex.n_cta1, 1))()
    arrs["cta2"] = (C.c_int32 * max(ex.n_cta2, 1))()
    for n in ("sta_mjobs", "psi_mjobs", "prod_mjobs"):
        arrs[n] = (OzJobC * max(getattr(ex, "n_" + n), 1))()
    arrs["prod_rows"] = (OzProwC * max(ex.n_prod_rows, 1))()
    for k, a in arrs.items():
        setattr(ex, k, C.cast(a, type(getattr(ex, k))))
    _chk(call(C.byref(ex)))
    return {"ex": ex, **arrs}
