"""The device path against the committed golden fixtures (tests/golden).

FP64 H*psi to 1e-12 and split-precision (5 slices) H*psi to 2e-9 of
max|H psi|, the device Lanczos energy to 1e-11 relative, and the device
truncation of the frozen ground state (kept count, truncation error,
entropies to 1e-10, kept sector shapes) -- all on the fingerprinted inputs.
"""
import os

import numpy as np
import pytest

from grand_sql_tj_b200 import synth
from tests.golden.make_golden import GOLDEN_CASES, fingerprint

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


@pytest.fixture(scope="module")
def ctxs(product_lib):
    from grand_sql_tj_b200.lib import TJ_PREC_OZAKI, Context
    f, o = Context(0), Context(0)
    o.set_precision(TJ_PREC_OZAKI, 5)
    yield f, o
    f.close()
    o.close()


@pytest.mark.parametrize("name,seed,kmin,kmax", GOLDEN_CASES)
def test_device_matches_golden(ctxs, name, seed, kmin, kmax):
    f, o = ctxs
    g = np.load(os.path.join(GOLD, "oracle_%s.npz" % name))
    sb = synth.workload(name, seed=seed)
    assert str(g["fingerprint"]) == fingerprint(sb), "synthetic inputs changed"
    ref = g["hpsi"]
    scale = np.max(np.abs(ref))
    assert np.max(np.abs(f.model_wave(sb).data - ref)) <= 1e-12 * scale
    assert np.max(np.abs(o.model_wave(sb).data - ref)) <= 2e-9 * scale
    e0, _, _ = f.lanczos_memo_new(sb, 1e-10)
    assert abs(e0 - float(g["e0"])) <= 1e-11 * max(1.0, abs(float(g["e0"])))
    psi = sb.wave.like(g["psi0"])
    r, blk = f.truncation(psi, 0, kmin, kmax, 1e-12)
    t = g["trunc"]
    assert r.num_state == int(t[0])
    assert np.allclose([r.trunc_err, r.entropy1, r.entropys], [t[1], t[2], t[4]], rtol=0, atol=1e-10)
    assert abs(r.entropy2 - t[3]) <= 1e-10
    shapes = np.array([[s.num_up, s.num_down, s.mat.shape[0], s.mat.shape[1]] for s in blk.subs])
    assert np.array_equal(shapes, g["trunc_sectors"])
