"""The split-precision (int8-slice) H*psi tables against the oracle, on the CPU.

tests/oz_exec.py executes the exported tables with the device's integer
arithmetic; the result must agree with the oracle's model_wave to the
accuracy of s truncated radix-128 slices, and every table index must stay
inside its pool.
"""
import numpy as np
import pytest

from grand_sql_tj_b200 import synth
from grand_sql_tj_b200.lib import TjError, ozaki_plan_export, plan_export
from tests.oz_exec import execute_ozaki


@pytest.mark.parametrize("name,slices,tol", [("tiny", 5, 2e-9), ("small", 5, 2e-9), ("small_gc", 4, 3e-7),
                                             ("cyl4", 5, 2e-9), ("cyl4", 6, 2e-11), ("cyl4", 8, 1e-13)])
def test_ozaki_tables_match_oracle(name, slices, tol, product_lib, oracle_lib):
    from oracle import oracle
    sb = synth.workload(name, seed=11)
    ref = oracle.model_wave(sb).data
    got = execute_ozaki(plan_export(sb), ozaki_plan_export(sb, slices), sb.wave.data)
    assert np.all(np.isfinite(got))
    err = np.max(np.abs(got - ref)) / np.max(np.abs(ref))
    assert err < tol, err


def test_ozaki_error_shrinks_with_slices(product_lib, oracle_lib):
    """Each extra slice buys about 7 bits (radix 128) until FP64 rounding."""
    from oracle import oracle
    sb = synth.workload("small", seed=2)
    ref = oracle.model_wave(sb).data
    plan = plan_export(sb)
    errs = []
    for s in (3, 4, 5):
        got = execute_ozaki(plan, ozaki_plan_export(sb, s), sb.wave.data)
        errs.append(np.max(np.abs(got - ref)) / np.max(np.abs(ref)))
    assert errs[0] > 20 * errs[1] > 400 * errs[2]


def test_ozaki_accounting(product_lib):
    sb = synth.workload("cyl4", seed=5)
    oz5 = ozaki_plan_export(sb, 5)["ex"]
    oz6 = ozaki_plan_export(sb, 6)["ex"]
    assert oz5.tile_n == 48 and oz6.tile_n == 32
    assert oz5.int8_ops > plan_export(sb)["ex"].flops   # padded int8 work exceeds the FP64 flops
    assert oz6.int8_ops > plan_export(sb)["ex"].flops
    assert oz5.n_items1 > 0 and oz5.n_items2 > 0 and oz5.n_sta_jobs > 0 and oz5.n_psi_jobs > 0
    assert oz5.rho0 < oz5.tau0 < oz5.pi0 < oz5.n_scales


def test_ozaki_rejects_bad_slice_count(product_lib):
    sb = synth.workload("tiny", seed=1)
    for s in (2, 9):
        with pytest.raises(TjError):
            ozaki_plan_export(sb, s)
