"""The oracle against the committed golden fixtures (tests/golden, made by
tests/golden/make_golden.py).

6j / 3j: the oracle's W6JS and W3JS restatements (block.f90:1508-1615, FP64
factorial table) against exact rational values, relative 1e-13, plus
closed-form special cases and the 6j orthogonality relation evaluated
directly.  Oracle results on seeded superblocks: model_wave, the Lanczos
energy and the truncation, against the frozen vectors (1e-12 relative), on
inputs whose fingerprint must equal the one recorded.
"""
import json
import math
import os

import numpy as np
import pytest

from grand_sql_tj_b200 import synth
from tests.golden.make_golden import GOLDEN_CASES, fingerprint

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


@pytest.fixture(scope="module")
def symbols():
    with open(os.path.join(GOLD, "w6j_w3j.json")) as f:
        return json.load(f)


def test_w6j_exact(oracle_lib, symbols):
    from oracle import oracle
    worst = 0.0
    for *j, v in symbols["w6j"]:
        got = oracle.w6js(*j)
        worst = max(worst, abs(got - v) / abs(v))
    assert worst <= 1e-13, worst


def test_w3j_exact(oracle_lib, symbols):
    from oracle import oracle
    worst = 0.0
    for *j, v in symbols["w3j"]:
        got = oracle.w3js(*j)
        worst = max(worst, abs(got - v) / abs(v))
    assert worst <= 1e-13, worst


def test_w6j_closed_forms_and_orthogonality(oracle_lib):
    from oracle import oracle
    # {a b c; 0 c b} = (-1)^(a+b+c) / sqrt((2b+1)(2c+1))   (doubled: (a+b+c)/2)
    for a in range(0, 9):
        for b in range(0, 9):
            for c in range(abs(a - b), a + b + 1, 2):
                want = (-1) ** ((a + b + c) // 2) / math.sqrt((b + 1) * (c + 1))
                assert abs(oracle.w6js(a, b, c, 0, c, b) - want) <= 1e-14
    # sum_x (2x+1)(2j+1) {a b x; c d j}{a b x; c d j'} = delta_jj'
    for (a, b, c, d) in [(2, 2, 2, 2), (3, 1, 3, 1), (4, 2, 3, 3), (5, 3, 4, 2)]:
        xs = range(abs(a - b), a + b + 1, 2)
        js = [j for j in range(0, 16) if (a + d + j) % 2 == 0 and abs(a - d) <= j <= a + d
              and abs(b - c) <= j <= b + c]
        for j in js:
            for k in js:
                s = sum((x + 1) * (j + 1) * oracle.w6js(a, b, x, c, d, j) * oracle.w6js(a, b, x, c, d, k) for x in xs)
                assert abs(s - (1.0 if j == k else 0.0)) <= 1e-13, (a, b, c, d, j, k, s)


@pytest.mark.parametrize("name,seed,kmin,kmax", GOLDEN_CASES)
def test_oracle_matches_frozen_results(oracle_lib, name, seed, kmin, kmax):
    from oracle import oracle
    g = np.load(os.path.join(GOLD, "oracle_%s.npz" % name))
    sb = synth.workload(name, seed=seed)
    assert str(g["fingerprint"]) == fingerprint(sb), "synthetic inputs changed"
    out = oracle.model_wave(sb).data
    assert np.max(np.abs(out - g["hpsi"])) <= 1e-12 * np.max(np.abs(g["hpsi"]))
    e0, iters, psi = oracle.lanczos(sb, 1e-10)
    assert abs(e0 - float(g["e0"])) <= 1e-12 * max(1.0, abs(float(g["e0"])))
    r, blk, ev = oracle.truncation(psi, 0, kmin, kmax, 1e-12)
    t = g["trunc"]
    assert r.num_state == int(t[0])
    assert np.allclose([r.trunc_err, r.entropy1, r.entropy2, r.entropys], t[1:], rtol=0, atol=1e-10)
    assert np.max(np.abs(np.sort(ev) - np.sort(g["rho_eigs"]))) <= 1e-12


def test_product_w6j_w3j_exact(product_lib, symbols):
    """The library's own 6j and 3j (the coefficient tables of every plan; the
    3j of block_mul_block_ndia) against the same exact rational values."""
    from grand_sql_tj_b200.lib import lib
    L = lib()
    w6 = max(abs(L.tj_w6js(*j) - v) / abs(v) for *j, v in symbols["w6j"])
    w3 = max(abs(L.tj_w3js(*j) - v) / abs(v) for *j, v in symbols["w3j"])
    assert w6 <= 1e-13 and w3 <= 1e-13, (w6, w3)
