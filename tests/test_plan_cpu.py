"""The H*psi compiler against the oracle, on the CPU.

The product compiles model_wave + hmerge into grouped-GEMM task lists; here
those lists are executed with numpy (tests/plan_exec.py) and compared with
the oracle's restatement of model_wave on the same seeded superblocks.
"""
import numpy as np
import pytest

from grand_sql_tj_b200 import synth
from grand_sql_tj_b200.lib import plan_export
from tests.plan_exec import execute, execute_items

CASES = ["tiny", "small", "small_gc", "cyl4"]


@pytest.mark.parametrize("name", CASES)
def test_plan_matches_oracle(name, product_lib, oracle_lib):
    from oracle import oracle
    sb = synth.workload(name, seed=11)
    ref = oracle.model_wave(sb).data
    plan = plan_export(sb)
    got = execute(plan, sb.wave.data)
    err = np.max(np.abs(got - ref)) / np.max(np.abs(ref))
    assert err < 1e-13, err


@pytest.mark.parametrize("name", ["small", "cyl4"])
def test_plan_random_vectors(name, product_lib, oracle_lib):
    """Linearity in psi: two random vectors and their sum."""
    from oracle import oracle
    sb = synth.workload(name, seed=3)
    rng = np.random.default_rng(7)
    plan = plan_export(sb)
    for _ in range(2):
        v = sb.wave.like(rng.standard_normal(sb.wave.dim))
        ref = oracle.model_wave(sb, v).data
        got = execute(plan, v.data)
        assert np.max(np.abs(got - ref)) <= 1e-13 * np.max(np.abs(ref))


def test_plan_accounting(product_lib):
    sb = synth.workload("cyl4", seed=5)
    ex = plan_export(sb)["ex"]
    assert ex.flops > 0 and ex.flops_ref >= ex.flops * 0.999
    assert ex.bytes >= 8 * 3 * sb.wave.dim
    assert ex.n_cells2 > 0 and ex.n_tasks2 > ex.n_cells2


@pytest.mark.parametrize("name", ["cyl4", "ladder16_m256"])
def test_plan_items_cover_every_cell(name, product_lib, oracle_lib):
    """Work items + reduce records (split-K) reproduce the oracle; every output entry is written once."""
    from oracle import oracle
    sb = synth.workload(name, seed=19)
    ref = oracle.model_wave(sb).data
    plan = plan_export(sb)
    got = execute_items(plan, sb.wave.data)
    assert np.all(np.isfinite(got))
    assert np.max(np.abs(got - ref)) <= 1e-13 * np.max(np.abs(ref))


@pytest.mark.parametrize("name", ["tiny", "small", "small_gc", "cyl4"])
def test_oracle_hpsi_is_symmetric(name, oracle_lib):
    """<x, H y> = <H x, y>: the synthetic operators obey the reduced Hermiticity
    rules, so every term's 6j weights and phases must pair up with those of
    its transposed partner (a wrong phase or 6j argument breaks the symmetry)."""
    from oracle import oracle
    sb = synth.workload(name, seed=4)
    rng = np.random.default_rng(0)
    x = sb.wave.like(rng.standard_normal(sb.wave.dim))
    y = sb.wave.like(rng.standard_normal(sb.wave.dim))
    hx, hy = oracle.model_wave(sb, x).data, oracle.model_wave(sb, y).data
    a, b = float(x.data @ hy), float(hx @ y.data)
    assert abs(a - b) <= 1e-14 * np.linalg.norm(hx) * np.linalg.norm(y.data)
