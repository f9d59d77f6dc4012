"""tj_model_wave_noalloc: H*psi for callers that cannot allocate device memory.

Such callers (a Fortran driver whose device memory comes from its own pool,
or a program that forbids allocation during a solve) hand the library their
own device buffers for the operators and the wavefunctions; the library's
scratch is a fixed array in device global memory.  This test copies a
superblock's operators and psi to device memory it owns, calls the
allocation-free entry point twice in a row through the C ABI, and checks each
result against the regular tj_model_wave (same 1e-12 relative tolerance as
the other H*psi tests).  It is collected last so that a failure here never
hides the rest of the suite.
"""
import ctypes as C

import numpy as np
import pytest

from grand_sql_tj_b200 import synth
from grand_sql_tj_b200.structs import TjBlock, TjBlockSet, TjModel, TjWave, c_double_p

pytestmark = pytest.mark.gpu


def _dev_block(pb, keep):
    import torch
    t = torch.from_numpy(pb.data.copy()).cuda()
    keep.append(t)
    c = pb.c
    return TjBlock(c.len, c.num, c.dim, c.up_dif, c.down_dif, 0, c.sub, C.cast(C.c_void_p(t.data_ptr()), c_double_p))


def _dev_model(pm, keep):
    n = pm.c.nsub
    sets = (TjBlockSet * max(n, 1))()
    for i in range(n):
        sets[i] = TjBlockSet(*[_dev_block(p, keep) for p in pm.sets[i]])
    keep.append(sets)
    return TjModel(pm.c.len, n, _dev_block(pm.ham, keep), C.cast(sets, C.POINTER(TjBlockSet)))


def test_model_wave_noalloc_matches_model_wave(product_lib):
    import torch
    from grand_sql_tj_b200.lib import Context, lib
    L = lib()
    L.tj_model_wave_noalloc.argtypes = [C.c_void_p] * 7 + [C.c_void_p]
    sb = synth.workload("cyl4", seed=31)
    ctx = Context(0)
    expected = ctx.model_wave(sb).data.copy()
    ctx.close()

    keep = []
    ps, pe = sb.sys.pack(), sb.env.pack()
    bs, be = sb.sys_bs.pack(), sb.env_bs.pack()
    dsys, denv = _dev_model(ps, keep), _dev_model(pe, keep)
    x = torch.from_numpy(sb.wave.data.copy()).cuda()
    y = torch.empty_like(x)
    w = sb.wave.c
    win = TjWave(w.sys_len, w.env_len, w.num, 0, w.dim, w.sub, C.cast(C.c_void_p(x.data_ptr()), c_double_p))
    wout = TjWave(w.sys_len, w.env_len, w.num, 0, w.dim, w.sub, C.cast(C.c_void_p(y.data_ptr()), c_double_p))
    torch.cuda.synchronize()
    scale = np.max(np.abs(expected))
    for call in range(2):
        y.fill_(float("nan"))
        torch.cuda.synchronize()
        rc = L.tj_model_wave_noalloc(C.addressof(sb.lat.c), C.addressof(dsys), C.addressof(denv),
                                     C.addressof(bs.c), C.addressof(be.c), C.addressof(win),
                                     C.addressof(wout), None)
        assert rc == 0, L.tj_last_error().decode()
        got = y.cpu().numpy()
        assert np.all(np.isfinite(got)), "call %d left unwritten entries" % call
        err = np.max(np.abs(got - expected)) / scale
        assert err < 1e-12, (call, err)


def test_model_wave_noalloc_rejects_overlapping_vectors(product_lib):
    """The second GEMM pass reads psi while other tiles already write H*psi, so
    an in-place call (outvec sharing invec's memory) would silently give wrong
    numbers; the entry point refuses it with TJ_ERR_ARG before any GPU work."""
    import torch
    from grand_sql_tj_b200.lib import lib
    L = lib()
    L.tj_model_wave_noalloc.argtypes = [C.c_void_p] * 7 + [C.c_void_p]
    sb = synth.workload("tiny", seed=5)
    keep = []
    ps, pe = sb.sys.pack(), sb.env.pack()
    bs, be = sb.sys_bs.pack(), sb.env_bs.pack()
    dsys, denv = _dev_model(ps, keep), _dev_model(pe, keep)
    x = torch.from_numpy(np.concatenate([sb.wave.data, sb.wave.data])).cuda()
    torch.cuda.synchronize()
    w = sb.wave.c
    base = x.data_ptr()
    for shift in (0, 8 * max(w.dim // 2, 1)):   # same buffer, and a partial overlap
        win = TjWave(w.sys_len, w.env_len, w.num, 0, w.dim, w.sub, C.cast(C.c_void_p(base), c_double_p))
        wout = TjWave(w.sys_len, w.env_len, w.num, 0, w.dim, w.sub, C.cast(C.c_void_p(base + shift), c_double_p))
        rc = L.tj_model_wave_noalloc(C.addressof(sb.lat.c), C.addressof(dsys), C.addressof(denv),
                                     C.addressof(bs.c), C.addressof(be.c), C.addressof(win),
                                     C.addressof(wout), None)
        assert rc == 1, (shift, rc)
        assert "overlap" in L.tj_last_error().decode()
