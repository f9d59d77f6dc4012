"""H*psi and Lanczos on the B200 against the oracle (FP64, bit-level algorithm parity).

Tolerances: H*psi elementwise relative error <= 1e-12 of max|H psi| (FP64
GEMMs in a different summation order); Lanczos energy |dE| <= 1e-9 |E| with
the same start vector and stopping threshold, Ritz-vector overlap >= 1 - 1e-8.
"""
import numpy as np
import pytest

from grand_sql_tj_b200 import synth

pytestmark = pytest.mark.gpu

CASES = ["tiny", "small", "small_gc", "cyl4"]


@pytest.fixture(scope="module")
def ctx(product_lib):
    from grand_sql_tj_b200.lib import Context
    c = Context(0)
    yield c
    c.close()


@pytest.mark.parametrize("name", CASES)
def test_model_wave(ctx, oracle_lib, name):
    from oracle import oracle
    sb = synth.workload(name, seed=21)
    ref = oracle.model_wave(sb).data
    got = ctx.model_wave(sb).data
    err = np.max(np.abs(got - ref)) / np.max(np.abs(ref))
    assert err < 1e-12, err


def test_model_wave_repeat_and_linearity(ctx, oracle_lib):
    """Two calls on the cached plan, and H(a x + y) = a H x + H y."""
    sb = synth.workload("cyl4", seed=2)
    rng = np.random.default_rng(1)
    x = sb.wave.like(rng.standard_normal(sb.wave.dim))
    y = sb.wave.like(rng.standard_normal(sb.wave.dim))
    hx = ctx.model_wave(sb, x).data
    hy = ctx.model_wave(sb, y).data
    hz = ctx.model_wave(sb, sb.wave.like(2.5 * x.data + y.data)).data
    assert np.max(np.abs(hz - (2.5 * hx + hy))) <= 1e-12 * np.max(np.abs(hz))
    assert np.array_equal(ctx.model_wave(sb, x).data, hx)   # deterministic


def test_model_wave_ladder16(ctx, oracle_lib):
    from oracle import oracle
    sb = synth.workload("ladder16_m256", seed=4)
    ref = oracle.model_wave(sb).data
    got = ctx.model_wave(sb).data
    assert np.max(np.abs(got - ref)) <= 1e-12 * np.max(np.abs(ref))


@pytest.mark.parametrize("name", ["small", "small_gc", "cyl4"])
def test_lanczos(ctx, oracle_lib, name):
    from oracle import oracle
    sb = synth.workload(name, seed=9)
    lz = 1e-10
    e_ref, it_ref, w_ref = oracle.lanczos(sb, lz)
    e, it, w = ctx.lanczos_memo_new(sb, lz)
    assert abs(e - e_ref) <= 1e-9 * abs(e_ref), (e, e_ref, it, it_ref)
    ov = abs(float(np.dot(w.data, w_ref.data)))
    assert ov >= 1 - 1e-8, ov
    assert abs(np.linalg.norm(w.data) - 1.0) < 1e-12


def test_lanczos_reference_threshold(ctx, oracle_lib):
    """The reference's sweep threshold lanzero = 2e-5 (eigen.f90 / main.f90:104,169)."""
    from oracle import oracle
    sb = synth.workload("cyl4", seed=13)
    lz = float(np.float32(20.0e-6))
    e_ref, it_ref, _ = oracle.lanczos(sb, lz)
    e, it, _ = ctx.lanczos_memo_new(sb, lz)
    assert it == it_ref
    assert abs(e - e_ref) <= 1e-10 * abs(e_ref)


def test_errors_are_reported(ctx):
    from grand_sql_tj_b200.lib import TjError
    sb = synth.workload("tiny", seed=1)
    bad = sb.wave.like()
    bad.sub[0].sys_dim = bad.sub[0].sys_dim + 1   # sector no longer matches the basis
    with pytest.raises(TjError):
        ctx.model_wave(sb, bad)
