"""Independent superblocks in shared launches (tj_model_wave_multi): every
instance's H*psi equals the one computed alone, in FP64 (1e-13 of max|H psi|;
only the split-K summation order may differ) and with 5 int8 slices (the
same splits and scales per instance: 1e-13 of max|H psi| against the
instance alone), and the cached merged plan gives the same result again."""
import numpy as np
import pytest

from grand_sql_tj_b200 import synth

pytestmark = pytest.mark.gpu

CASES = [("small", 3), ("cyl4", 4), ("tiny", 5), ("small_gc", 6)]


@pytest.mark.parametrize("prec", [0, 1])
def test_multi_equals_single(product_lib, prec):
    from grand_sql_tj_b200.lib import TJ_PREC_OZAKI, Context
    sbs = [synth.workload(n, seed=s) for n, s in CASES]
    c = Context(0)
    try:
        if prec:
            c.set_precision(TJ_PREC_OZAKI, 5)
        singles = [c.model_wave(sb).data for sb in sbs]
        outs, _ = c.model_wave_multi(sbs)
        for a, b in zip(outs, singles):
            assert np.max(np.abs(a.data - b)) <= 1e-13 * np.max(np.abs(b))
        again, ms = c.model_wave_multi(sbs, reps=3)
        assert ms > 0
        for a, b in zip(again, outs):
            assert np.max(np.abs(a.data - b.data)) <= 1e-13 * np.max(np.abs(b.data))
    finally:
        c.close()
