"""Split-precision H*psi (int8 slices on the tcgen05 tensor cores) on the B200.

The device result must equal the numpy execution of the same tables
(tests/oz_exec.py: identical integer products, the same FP64 epilogue order)
to FP64 rounding, and the oracle's FP64 model_wave to the accuracy of the
slices: <= 2e-9 of max|H psi| with 5 slices, <= 1e-12 with 7.  The ground
state energy from Lanczos over split-precision H*psi must agree with the
FP64 one to |dE| per site <= 1e-9.
"""
import numpy as np
import pytest

from grand_sql_tj_b200 import synth

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx(product_lib):
    from grand_sql_tj_b200.lib import TJ_PREC_OZAKI, Context
    c = Context(0)
    c.set_precision(TJ_PREC_OZAKI, 5)
    yield c
    c.close()


@pytest.mark.parametrize("name", ["tiny", "small", "small_gc", "cyl4"])
def test_ozaki_matches_tables_and_oracle(ctx, oracle_lib, name):
    from oracle import oracle
    from grand_sql_tj_b200.lib import ozaki_plan_export, plan_export
    from tests.oz_exec import execute_ozaki
    sb = synth.workload(name, seed=21)
    ref = oracle.model_wave(sb).data
    got = ctx.model_wave(sb).data
    emu = execute_ozaki(plan_export(sb), ozaki_plan_export(sb, 5), sb.wave.data)
    scale = np.max(np.abs(ref))
    assert np.max(np.abs(got - emu)) <= 1e-14 * scale
    assert np.max(np.abs(got - ref)) <= 2e-9 * scale


def test_ozaki_deterministic_and_linear(ctx):
    sb = synth.workload("cyl4", seed=2)
    rng = np.random.default_rng(1)
    x = sb.wave.like(rng.standard_normal(sb.wave.dim))
    y = sb.wave.like(rng.standard_normal(sb.wave.dim))
    hx = ctx.model_wave(sb, x).data
    hy = ctx.model_wave(sb, y).data
    hz = ctx.model_wave(sb, sb.wave.like(2.5 * x.data + y.data)).data
    assert np.array_equal(ctx.model_wave(sb, x).data, hx)
    assert np.max(np.abs(hz - (2.5 * hx + hy))) <= 4e-9 * np.max(np.abs(hz))


def test_ozaki_seven_slices(product_lib, oracle_lib):
    from oracle import oracle
    from grand_sql_tj_b200.lib import TJ_PREC_OZAKI, Context
    sb = synth.workload("ladder16_m256", seed=4)
    ref = oracle.model_wave(sb).data
    c = Context(0)
    try:
        c.set_precision(TJ_PREC_OZAKI, 7)
        got = c.model_wave(sb).data
        assert c.stats().int8_ops > 0
    finally:
        c.close()
    assert np.max(np.abs(got - ref)) <= 1e-12 * np.max(np.abs(ref))


def test_ozaki_lanczos_energy_per_site(ctx, product_lib):
    from grand_sql_tj_b200.lib import Context
    sb = synth.workload("cyl4", seed=9)
    f = Context(0)
    try:
        e64, _, w64 = f.lanczos_memo_new(sb, 1e-10)
    finally:
        f.close()
    e, _, w = ctx.lanczos_memo_new(sb, 1e-10)
    nsite = sb.geo.num_site
    assert abs(e - e64) / nsite <= 1e-9, (e, e64)
    assert abs(float(np.dot(w.data, w64.data))) >= 1 - 1e-7


def test_ozaki_long_families_in_pieces(product_lib):
    """6x24 m=6000: families longer than one int32 accumulation (about 26k
    inner dimension at 5 slices) are accumulated in pieces; 7 slices must
    reproduce the FP64 device result to 1e-12 of max|H psi|."""
    from grand_sql_tj_b200.lib import TJ_PREC_OZAKI, Context
    sb = synth.workload("cyl6x24_m6000", seed=8)
    f, o = Context(0), Context(0)
    try:
        o.set_precision(TJ_PREC_OZAKI, 7)
        ref = f.model_wave(sb).data
        got = o.model_wave(sb).data
    finally:
        f.close()
        o.close()
    assert np.max(np.abs(got - ref)) <= 1e-12 * np.max(np.abs(ref))
