"""Failure paths on the B200, made without faulting the GPU.

  * A NaN in psi, or an infinity in an operator, cannot be split into int8
    digits: the split-precision path reports TJ_ERR_NUMERIC (the maximum
    kernel flags any non-finite value it reads) instead of returning a
    silently wrong product; the FP64 path lets the NaN propagate into H*psi
    as the reference's DGEMMs do, and Lanczos reports TJ_ERR_NUMERIC on the
    non-finite beta.
  * The split-precision GEMM's pipeline waits are bounded: with the bound
    set to 0 s (tj_set_wait_limit) its first wait that is not already
    satisfied gives up, the kernel drains its copies and MMAs in flight
    (with their own 2 s bound), frees its tensor memory and returns, and the
    call returns TJ_ERR_TIMEOUT.
  * After each failure the same context, and a fresh one, compute H*psi
    that matches the oracle (2e-9 of max|H psi| with 5 slices).
"""
import numpy as np
import pytest

from grand_sql_tj_b200 import synth

pytestmark = pytest.mark.gpu


def _check(ctx, sb, ref):
    got = ctx.model_wave(sb).data
    assert np.max(np.abs(got - ref)) <= 2e-9 * np.max(np.abs(ref))


@pytest.fixture(scope="module")
def case(product_lib, oracle_lib):
    from oracle import oracle
    sb = synth.workload("cyl4", seed=23)
    return sb, oracle.model_wave(sb).data


def test_nan_in_psi(case):
    from grand_sql_tj_b200.lib import TJ_PREC_OZAKI, Context, TjError
    sb, ref = case
    bad = sb.wave.copy()
    bad.data[bad.dim // 3] = np.nan
    c = Context(0)
    try:
        c.set_precision(TJ_PREC_OZAKI, 5)
        with pytest.raises(TjError) as e:
            c.model_wave(sb, bad)
        assert e.value.code == 7
        _check(c, sb, ref)                      # the next call is clean
        c.set_precision(0, 5)                   # FP64: the NaN propagates, the call succeeds
        out = c.model_wave(sb, bad).data
        assert np.isnan(out).any()
        with pytest.raises(TjError) as e:
            c.lanczos_memo_new(sb, 1e-8, start=bad)
        assert e.value.code == 7
    finally:
        c.close()


def test_inf_in_operator(case):
    from grand_sql_tj_b200.lib import TJ_PREC_OZAKI, Context, TjError
    sb, ref = case
    sub = sb.sys.ham.subs[0]
    keep = sub.mat[0, 0]
    sub.mat[0, 0] = np.inf
    c = Context(0)
    try:
        c.set_precision(TJ_PREC_OZAKI, 5)
        with pytest.raises(TjError) as e:
            c.model_wave(sb)
        assert e.value.code == 7
    finally:
        sub.mat[0, 0] = keep
    try:
        c.step_begin()
        _check(c, sb, ref)
    finally:
        c.close()


def test_wait_bound_runs_out(case):
    from grand_sql_tj_b200.lib import TJ_PREC_OZAKI, Context, TjError
    sb, ref = case
    c = Context(0)
    try:
        c.set_precision(TJ_PREC_OZAKI, 5)
        _check(c, sb, ref)
        c.set_wait_limit(0.0)
        with pytest.raises(TjError) as e:
            c.model_wave(sb)
        assert e.value.code == 6
        c.set_wait_limit(2.0)
        _check(c, sb, ref)
    finally:
        c.close()
    fresh = Context(0)
    try:
        fresh.set_precision(TJ_PREC_OZAKI, 5)
        _check(fresh, sb, ref)
    finally:
        fresh.close()
