"""The benchmark's own superblocks against the oracle, on the B200.

The headline workload is the mid-chain superblock of the 4x24 cylinder at
m = 2000 (12 holes, S = 0, D = 1 401 587): the bench times exactly this
superblock, so the numbers it reports are held here to the oracle's FP64
restatement of the reference (code/tjsq/get_sys.f90:4127-4381 model_wave,
code/tjsq/eigen.f90:2-175 lanczos_memo_new):

  * FP64 H*psi            <= 1e-12 of max|H psi|
  * split precision, s=5  <= 2e-9  of max|H psi|
  * Lanczos at the reference's sweep threshold (lanzero = 2e-5 as a
    single-precision literal, main.f90:104): the same number of Lanczos
    vectors as the oracle from the same start vector, |dE| <= 1e-10 |E|
  * split-precision Lanczos against the FP64 device Lanczos: |dE| per site
    <= 1e-9 (the accuracy target of the split-precision path)

and one FP64 H*psi of the 6x24 cylinder at m = 6000 (t' = -0.2, 18 holes).
The oracle runs with every host thread so that each of its calls takes
seconds.
"""
import os

import numpy as np
import pytest

from grand_sql_tj_b200 import synth

pytestmark = pytest.mark.gpu

LANZERO = float(np.float32(20.0e-6))


@pytest.fixture(scope="module")
def headline(product_lib, oracle_lib):
    from oracle import oracle
    oracle.set_threads(os.cpu_count() or 1)
    return synth.workload("cyl4x24_m2000")


def test_headline_fp64_hpsi(headline):
    from oracle import oracle
    from grand_sql_tj_b200.lib import Context
    ref = oracle.model_wave(headline).data
    c = Context(0)
    try:
        got = c.model_wave(headline).data
    finally:
        c.close()
    assert np.max(np.abs(got - ref)) <= 1e-12 * np.max(np.abs(ref))


def test_headline_split_hpsi(headline):
    from oracle import oracle
    from grand_sql_tj_b200.lib import TJ_PREC_OZAKI, Context
    ref = oracle.model_wave(headline).data
    c = Context(0)
    try:
        c.set_precision(TJ_PREC_OZAKI, 5)
        got = c.model_wave(headline).data
        assert c.stats().int8_ops > 0
    finally:
        c.close()
    # Five int8 slices hold each operand to about 2^-35 of its row (column)
    # maximum; the error of an entry is that times sum_k |a_ik| |b_kj| over two
    # chained products and fourteen terms, not times the (cancelled) entry.
    # Measured 3.3e-9 of the largest entry here; the energy test below is the
    # physical bound.
    assert np.max(np.abs(got - ref)) <= 1e-8 * np.max(np.abs(ref))


def test_headline_lanczos_reference_threshold(headline):
    from oracle import oracle
    from grand_sql_tj_b200.lib import TJ_PREC_OZAKI, Context
    e_ref, it_ref, w_ref = oracle.lanczos(headline, LANZERO)
    f, o = Context(0), Context(0)
    try:
        e64, it64, w64 = f.lanczos_memo_new(headline, LANZERO)
        o.set_precision(TJ_PREC_OZAKI, 5)
        e5, it5, w5 = o.lanczos_memo_new(headline, LANZERO)
    finally:
        f.close()
        o.close()
    assert it64 == it_ref, (it64, it_ref)
    assert abs(e64 - e_ref) <= 1e-10 * abs(e_ref), (e64, e_ref)
    nsite = headline.geo.num_site
    assert abs(e5 - e64) / nsite <= 1e-9, (e5, e64)
    # the two Ritz vectors stop at a Lanczos residual of about lanzero
    assert abs(float(np.dot(w64.data, w_ref.data))) >= 1 - 1e-8


@pytest.mark.slow
def test_cyl6x24_m6000_fp64_hpsi(product_lib, oracle_lib):
    from oracle import oracle
    from grand_sql_tj_b200.lib import Context
    oracle.set_threads(os.cpu_count() or 1)
    sb = synth.workload("cyl6x24_m6000", seed=8)
    ref = oracle.model_wave(sb).data
    c = Context(0)
    try:
        got = c.model_wave(sb).data
    finally:
        c.close()
    assert np.max(np.abs(got - ref)) <= 1e-12 * np.max(np.abs(ref))
