"""ctypes wrapper of the CPU oracle (TEST INFRASTRUCTURE).

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg import
this module.  It loads oracle/liboracle_tj.so (built by `make -C oracle`),
which restates the tjsq Fortran hot path in C, and binds dgemm/dsyev/dstev
from the OpenBLAS bundled with scipy.  Parity is unpinned: see oracle_tj.h.
"""
from __future__ import annotations

import ctypes as C
import glob
import os
import subprocess

import numpy as np

from grand_sql_tj_b200.structs import (TjBasis, TjBlock, TjBlockResult, TjChain, TjLattice, TjModel, TjModelResult,
                                       TjTruncResult, TjWave, TjBlockSub, Block, block_from_c_result,
                                       call_block_result, call_model_result)

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "liboracle_tj.so")


def build(force: bool = False) -> str:
    src = [os.path.join(HERE, f) for f in ("oracle_tj.c", "oracle_tj.h")]
    if force or not os.path.exists(LIB) or any(os.path.getmtime(s) > os.path.getmtime(LIB) for s in src):
        subprocess.run(["make", "-s", "-C", HERE, "-B" if force else "liboracle_tj.so"], check=True)
    return LIB


def openblas_path() -> str:
    import scipy
    d = os.path.join(os.path.dirname(os.path.dirname(scipy.__file__)), "scipy.libs")
    cands = sorted(glob.glob(os.path.join(d, "libscipy_openblas*.so")))
    if not cands:
        raise RuntimeError("scipy's bundled OpenBLAS not found")
    return cands[0]


_lib = None


def lib(threads: int = 1):
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            build()
        L = C.CDLL(LIB)
        P = C.POINTER
        L.ora_init.argtypes = [C.c_char_p, C.c_int]
        L.ora_set_threads.argtypes = [C.c_int]
        L.ora_w6js.restype = C.c_double
        L.ora_w6js.argtypes = [C.c_int] * 6
        L.ora_w3js.restype = C.c_double
        L.ora_w3js.argtypes = [C.c_int] * 6
        L.ora_model_wave.argtypes = [P(TjLattice), P(TjModel), P(TjModel), P(TjBasis), P(TjBasis),
                                     P(TjWave), P(TjWave)]
        L.ora_lanczos.argtypes = [P(TjLattice), P(TjModel), P(TjModel), P(TjBasis), P(TjBasis),
                                  P(TjWave), C.c_double, P(C.c_double), P(C.c_int)]
        L.ora_truncation.argtypes = [P(TjWave), C.c_int, C.c_int, C.c_int, C.c_double,
                                     P(TjTruncResult), P(C.c_double)]
        L.ora_last_error.restype = C.c_char_p
        for n in ("ora_measure_sys_block", "ora_measure_env_block"):
            getattr(L, n).argtypes = [P(TjBlock), P(TjBasis), P(TjWave), P(C.c_double)]
        L.ora_sys_block_env_block_cor_dia.argtypes = [P(TjBlock), P(TjBlock), P(TjBasis), P(TjBasis),
                                                      P(TjWave), P(C.c_double)]
        for n in ("ora_sys_block_env_block_cor_ndia", "ora_sys_block_env_site_cor_ndia",
                  "ora_sys_site_env_block_cor_ndia", "ora_sys_site_env_site_cor_ndia"):
            getattr(L, n).argtypes = [P(TjBlock), P(TjBlock), P(TjBasis), P(TjBasis), P(TjWave),
                                      C.c_char, P(C.c_double)]
        for n in ("ora_sys_block_site_cor_ndia", "ora_env_block_site_cor_ndia"):
            getattr(L, n).argtypes = [P(TjBlock), P(TjBlock), P(TjBasis), P(TjWave), C.c_char,
                                      P(C.c_double)]
        L.ora_get_hamiltonian.argtypes = [P(TjLattice), C.c_int, C.c_int, P(TjModel), P(TjBasis), P(TjBlock),
                                          P(TjModelResult)]
        L.ora_wave_trans.argtypes = [C.c_int, P(TjBasis), P(TjBasis), P(TjBlock), P(TjBlock), P(TjWave), P(TjWave)]
        L.ora_get_oper.argtypes = [C.c_int, C.c_int, P(TjChain), P(TjBlock), C.c_int, C.c_int, C.c_int, C.c_char,
                                   P(TjBlockResult)]
        L.ora_change_oper.argtypes = L.ora_get_oper.argtypes
        L.ora_block_mul_block_ndia.argtypes = [P(TjBlock), C.c_char, P(TjBlock), C.c_char, C.c_double, C.c_int,
                                               P(TjBasis), P(TjBlockResult)]
        L.ora_update_trun.argtypes = [C.c_int, P(TjBlock), P(TjBlock), P(TjBlockResult)]
        L.ora_site_operator.argtypes = [C.c_int, C.c_int, P(TjBlock), P(TjBlockSub), P(C.c_double)]
        rc = L.ora_init(openblas_path().encode(), threads)
        if rc:
            raise RuntimeError("ora_init failed: " + L.ora_last_error().decode())
        _lib = L
    return _lib


def set_threads(n: int) -> None:
    lib().ora_set_threads(n)


def _chk(rc):
    if rc:
        raise RuntimeError("oracle error %d: %s" % (rc, lib().ora_last_error().decode()))


def w6js(*a) -> float:
    return lib().ora_w6js(*a)


def w3js(*a) -> float:
    return lib().ora_w3js(*a)


def model_wave(sb, invec=None):
    """hmerge + model_wave on a synth.Superblock; returns the output Wave."""
    L = lib()
    invec = sb.wave if invec is None else invec
    ps, pe = sb.sys.pack(), sb.env.pack()
    bs, be = sb.sys_bs.pack(), sb.env_bs.pack()
    out = invec.like()
    _chk(L.ora_model_wave(C.byref(sb.lat.c), C.byref(ps.c), C.byref(pe.c), C.byref(bs.c),
                          C.byref(be.c), C.byref(invec.c), C.byref(out.c)))
    return out


def lanczos(sb, lanzero: float, start=None):
    L = lib()
    w = (sb.wave if start is None else start).copy()
    ps, pe = sb.sys.pack(), sb.env.pack()
    bs, be = sb.sys_bs.pack(), sb.env_bs.pack()
    e, it = C.c_double(), C.c_int()
    _chk(L.ora_lanczos(C.byref(sb.lat.c), C.byref(ps.c), C.byref(pe.c), C.byref(bs.c), C.byref(be.c),
                       C.byref(w.c), lanzero, C.byref(e), C.byref(it)))
    return e.value, it.value, w


def truncation(wave, side: int, kept_min: int, kept_max: int, trun_err: float):
    """Returns (result struct, trun_op Block, per-sector eigenvalues)."""
    L = lib()
    r = TjTruncResult()
    _chk(L.ora_truncation(C.byref(wave.c), side, kept_min, kept_max, trun_err, C.byref(r), None))
    subs = (TjBlockSub * max(r.num, 1))()
    data = np.zeros(max(r.data_len, 1))
    ndim = sum((s.sys_dim if side == 0 else s.env_dim) for s in wave.sectors)
    ev = np.zeros(max(ndim, 1))
    r.sub = C.cast(subs, C.POINTER(TjBlockSub))
    r.data = data.ctypes.data_as(C.POINTER(C.c_double))
    _chk(L.ora_truncation(C.byref(wave.c), side, kept_min, kept_max, trun_err, C.byref(r),
                          ev.ctypes.data_as(C.POINTER(C.c_double))))
    length = wave.sys_len if side == 0 else wave.env_len
    return r, block_from_c_result(r, length, subs, data), ev[:ndim]


def site_operator(which: int, up_bias: int) -> Block:
    from grand_sql_tj_b200.structs import SubBlock
    L = lib()
    b = TjBlock()
    subs = (TjBlockSub * 2)()
    vals = (C.c_double * 2)()
    n = L.ora_site_operator(which, up_bias, C.byref(b), subs, vals)
    return Block(1, b.up_dif, b.down_dif,
                 [SubBlock(subs[i].num_up, subs[i].num_down, subs[i].down_dif,
                           np.array([[vals[i]]], order="F")) for i in range(n)])


def correlator(name: str, a, b, sys_bs, env_bs, wave, flag: str = "B") -> float:
    """name is the reference routine name, e.g. 'sys_block_env_block_cor_ndia'."""
    L = lib()
    v = C.c_double()
    pa = a.pack()
    pb = b.pack() if b is not None else None
    ps = sys_bs.pack() if sys_bs is not None else None
    pe = env_bs.pack() if env_bs is not None else None
    fn = getattr(L, "ora_" + name)
    f = flag.encode()
    if name == "measure_sys_block":
        _chk(fn(C.byref(pa.c), C.byref(ps.c), C.byref(wave.c), C.byref(v)))
    elif name == "measure_env_block":
        _chk(fn(C.byref(pa.c), C.byref(pe.c), C.byref(wave.c), C.byref(v)))
    elif name == "sys_block_env_block_cor_dia":
        _chk(fn(C.byref(pa.c), C.byref(pb.c), C.byref(ps.c), C.byref(pe.c), C.byref(wave.c), C.byref(v)))
    elif name == "sys_block_site_cor_ndia":
        _chk(fn(C.byref(pa.c), C.byref(pb.c), C.byref(ps.c), C.byref(wave.c), f, C.byref(v)))
    elif name == "env_block_site_cor_ndia":
        _chk(fn(C.byref(pa.c), C.byref(pb.c), C.byref(pe.c), C.byref(wave.c), f, C.byref(v)))
    else:
        _chk(fn(C.byref(pa.c), C.byref(pb.c), C.byref(ps.c), C.byref(pe.c), C.byref(wave.c), f, C.byref(v)))
    return v.value


def get_hamiltonian(lat, side: int, mshift: int, pre, basis, trun):
    """Get_Hamiltonian_Sys (side 0) / Get_Hamiltonian_Env (side 1): the block
    `pre` enlarged into `basis` and truncated with the Block `trun`; returns the
    new Model."""
    L = lib()
    pp, pb, pt = pre.pack(), basis.pack(), trun.pack()
    rc, m = call_model_result(lambda r: L.ora_get_hamiltonian(C.byref(lat.c), side, mshift, C.byref(pp.c),
                                                              C.byref(pb.c), C.byref(pt.c), r))
    _chk(rc)
    return m


def lanczos_parts(lat, sys, env, sys_bs, env_bs, wave, lanzero: float):
    """lanczos_memo_new on explicit models and bases; `wave` is the start vector (copied)."""
    L = lib()
    w = wave.copy()
    ps, pe = sys.pack(), env.pack()
    bs, be = sys_bs.pack(), env_bs.pack()
    e, it = C.c_double(), C.c_int()
    _chk(L.ora_lanczos(C.byref(lat.c), C.byref(ps.c), C.byref(pe.c), C.byref(bs.c), C.byref(be.c),
                       C.byref(w.c), lanzero, C.byref(e), C.byref(it)))
    return e.value, it.value, w


def wave_trans(direction: int, sys_bs, env_bs, sys_trun, env_trun, old, new_wave):
    """wave_trans_LR (direction 0) / wave_trans_RL (direction 1): fills and returns
    `new_wave` (a Wave with the next superblock's sectors)."""
    L = lib()
    pb, pe, ps, pt = sys_bs.pack(), env_bs.pack(), sys_trun.pack(), env_trun.pack()
    _chk(L.ora_wave_trans(direction, C.byref(pb.c), C.byref(pe.c), C.byref(ps.c), C.byref(pt.c), C.byref(old.c),
                          C.byref(new_wave.c)))
    return new_wave


def get_oper(side, dia, chain, st_oper, old_idx, new_idx, truns, types="B"):
    """Get_{sys,env}_oper_{dia,ndia}: chain is a structs.PackedChain."""
    L = lib()
    ps = st_oper.pack()
    rc, b = call_block_result(lambda r: L.ora_get_oper(side, int(dia), C.byref(chain.c), C.byref(ps.c), old_idx,
                                                       new_idx, int(truns), types.encode(), r))
    _chk(rc)
    return b


def change_oper(side, dia, chain, old_oper, old_idx, new_idx, truns, types="B"):
    """Change_{sys,env}_oper_{dia,ndia}."""
    L = lib()
    ps = old_oper.pack()
    rc, b = call_block_result(lambda r: L.ora_change_oper(side, int(dia), C.byref(chain.c), C.byref(ps.c), old_idx,
                                                          new_idx, int(truns), types.encode(), r))
    _chk(rc)
    return b


def block_mul_block_ndia(o1, f1, o2, f2, coef, down_dif, basis):
    L = lib()
    p1, p2, pb = o1.pack(), o2.pack(), basis.pack()
    rc, b = call_block_result(lambda r: L.ora_block_mul_block_ndia(C.byref(p1.c), f1.encode(), C.byref(p2.c),
                                                                   f2.encode(), coef, down_dif, C.byref(pb.c), r))
    _chk(rc)
    return b


def update_trun(dia, ori, trun):
    L = lib()
    po, pt = ori.pack(), trun.pack()
    rc, b = call_block_result(lambda r: L.ora_update_trun(int(dia), C.byref(po.c), C.byref(pt.c), r))
    _chk(rc)
    return b


class OracleBackend:
    """The hot-path calls of grand_sql_tj_b200.sweep.Dmrg on the oracle (CPU)."""

    def lanczos(self, lat, sys, env, sys_bs, env_bs, wave, lanzero):
        return lanczos_parts(lat, sys, env, sys_bs, env_bs, wave, lanzero)

    def truncation(self, wave, side, kept_min, kept_max, trun_err):
        r, trun, _ = truncation(wave, side, kept_min, kept_max, trun_err)
        return r, trun

    def get_hamiltonian(self, lat, side, mshift, pre, basis, trun):
        return get_hamiltonian(lat, side, mshift, pre, basis, trun)

    def wave_trans(self, direction, sys_bs, env_bs, sys_trun, env_trun, old, new_wave):
        return wave_trans(direction, sys_bs, env_bs, sys_trun, env_trun, old, new_wave)

    def get_oper(self, side, dia, chain, st_oper, old_idx, new_idx, truns, types="B"):
        return get_oper(side, dia, chain, st_oper, old_idx, new_idx, truns, types)

    def change_oper(self, side, dia, chain, old_oper, old_idx, new_idx, truns, types="B"):
        return change_oper(side, dia, chain, old_oper, old_idx, new_idx, truns, types)

    def block_mul_block_ndia(self, o1, f1, o2, f2, coef, down_dif, basis):
        return block_mul_block_ndia(o1, f1, o2, f2, coef, down_dif, basis)

    def update_trun(self, dia, ori, trun):
        return update_trun(dia, ori, trun)

    def correlator(self, name, a, b, sys_bs, env_bs, wave, flag="B"):
        return correlator(name, a, b, sys_bs, env_bs, wave, flag)
