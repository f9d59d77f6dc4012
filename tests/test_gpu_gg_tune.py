"""Grouped block-GEMM benchmark and the autotuner on the B200.

tj_grouped_gemm_bench: the one-launch grouped form, the one-launch-per-block
form and the autotuned grouped form all equal the numpy reference to 1e-12
of max|Y| (FP64; only the summation order differs).  tj_autotune: the
chosen tiling is one of the candidates, is cached for the histogram, and the
H*psi computed with it still equals the oracle to 1e-12 (FP64) / 2e-9 (5
slices).
"""
import numpy as np
import pytest

from grand_sql_tj_b200 import gg, synth

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx(product_lib):
    from grand_sql_tj_b200.lib import Context
    c = Context(0)
    yield c
    c.close()


def test_grouped_batch_matches_reference(ctx):
    b = gg.make_batch(n_cells=24, dmax=256, seed=3, pool_len=1 << 21)
    ref = gg.reference(b)
    scale = max(np.max(np.abs(v)) for v in ref.values())
    for mode in (0, 1, 2):
        ms, out, fl, tr = ctx.grouped_gemm_bench(b, mode, reps=2)
        assert ms > 0 and abs(fl - b.flops) < 1.0
        for c, y in ref.items():
            assert np.max(np.abs(gg.cell_view(b, out, c) - y)) <= 1e-12 * scale, (mode, c)
        if mode == 2:
            assert tr.items_per_cta in (3, 6, 12) and tr.min_ksteps in (128, 256, 512) and tr.ctas_per_sm in (2, 3, 4)
            assert tr.evaluated >= 7 and tr.tuned_ms <= tr.default_ms


@pytest.mark.parametrize("prec", [0, 1])
def test_autotune_hpsi(product_lib, oracle_lib, prec):
    from oracle import oracle
    from grand_sql_tj_b200.lib import TJ_PREC_OZAKI, TJ_TUNE_CACHED, Context
    sb = synth.workload("cyl4", seed=13)
    ref = oracle.model_wave(sb).data
    c = Context(0)
    try:
        if prec:
            c.set_precision(TJ_PREC_OZAKI, 5)
        tr = c.autotune(sb)
        assert tr.evaluated >= 3 and tr.tuned_ms <= tr.default_ms and tr.hist_key != 0
        if prec:
            assert tr.oz_bn in (32, 48) and tr.oz_item_cost in (2, 4, 8)
        got = c.model_wave(sb).data
        tol = 2e-9 if prec else 1e-12
        assert np.max(np.abs(got - ref)) <= tol * np.max(np.abs(ref))
        # a second context finds the stored choice for the same histogram
        d = Context(0)
        try:
            if prec:
                d.set_precision(TJ_PREC_OZAKI, 5)
            d.set_autotune(TJ_TUNE_CACHED)
            assert np.max(np.abs(d.model_wave(sb).data - got)) <= 1e-14 * np.max(np.abs(ref))
        finally:
            d.close()
    finally:
        c.close()
