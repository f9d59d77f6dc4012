"""Generates the golden fixtures of tests/golden (run from the repository root).

    python tests/golden/make_golden.py

w6j_w3j.json -- exact Wigner 6j and 3j symbols for all admissible doubled
spins up to 6, plus 600 seeded 6j symbols with doubled spins up to 24 (the
multiplet spins of m = 2000 blocks), from Racah's closed formulas evaluated in
rational arithmetic (fractions.Fraction; the square root taken in 50-digit
decimal), independent of the floating-point factorial table that W6JS and
W3JS (code/tjsq/block.f90:1508-1615) use.

oracle_<workload>.npz -- the oracle's FP64 results on seeded synthetic
superblocks, frozen: model_wave (hmerge + model_wave, get_sys.f90:4127-4593)
of the workload's wave, the Lanczos ground energy and iteration count at
lanzero = 1e-10 (eigen.f90:2-175), and the system-block truncation
(den_mat.f90:84-383) of that ground state.  A fingerprint (SHA-256 of the
inputs) makes a change of the synthetic generator fail loudly instead of
comparing different inputs.
"""
import hashlib
import json
import os
import sys
from decimal import Decimal, getcontext
from fractions import Fraction
from math import factorial

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

getcontext().prec = 50


def _fr(n):
    return Fraction(factorial(n)) if n >= 0 else None


def _delta2(a, b, c):
    """Triangle coefficient squared for doubled spins a, b, c (None if not a triad)."""
    if (a + b + c) % 2 or c > a + b or c < abs(a - b):
        return None
    return _fr((a + b - c) // 2) * _fr((a - b + c) // 2) * _fr((-a + b + c) // 2) / _fr((a + b + c) // 2 + 1)


def _signed_sqrt(square: Fraction, sign: int) -> float:
    if square == 0:
        return 0.0
    v = (Decimal(square.numerator) / Decimal(square.denominator)).sqrt()
    return float(v) * sign


def w6j_exact(j1, j2, j3, l1, l2, l3) -> float:
    """{j1 j2 j3; l1 l2 l3} on doubled spins, Racah's formula in rationals."""
    tri = [_delta2(j1, j2, j3), _delta2(j1, l2, l3), _delta2(l1, j2, l3), _delta2(l1, l2, j3)]
    if any(t is None for t in tri):
        return 0.0
    a = [(j1 + j2 + j3) // 2, (j1 + l2 + l3) // 2, (l1 + j2 + l3) // 2, (l1 + l2 + j3) // 2]
    b = [(j1 + j2 + l1 + l2) // 2, (j2 + j3 + l2 + l3) // 2, (j3 + j1 + l3 + l1) // 2]
    s = Fraction(0)
    for t in range(max(a), min(b) + 1):
        den = 1
        for x in a:
            den *= factorial(t - x)
        for y in b:
            den *= factorial(y - t)
        s += Fraction((-1) ** t * factorial(t + 1), den)
    pref = tri[0] * tri[1] * tri[2] * tri[3]
    return _signed_sqrt(pref * s * s, 1 if s > 0 else -1)


def w3j_exact(j1, j2, j3, m1, m2, m3) -> float:
    """(j1 j2 j3; m1 m2 m3) on doubled spins and projections, Racah's formula in rationals."""
    if m1 + m2 + m3 != 0:
        return 0.0
    d = _delta2(j1, j2, j3)
    if d is None:
        return 0.0
    for j, m in ((j1, m1), (j2, m2), (j3, m3)):
        if abs(m) > j or (j + m) % 2:
            return 0.0
    h = lambda x: x // 2
    pre = d
    for j, m in ((j1, m1), (j2, m2), (j3, m3)):
        pre *= _fr(h(j + m)) * _fr(h(j - m))
    s = Fraction(0)
    for k in range(0, h(j1 + j2 + j3) + 1):
        args = [k, h(j3 - j2 + m1) + k, h(j3 - j1 - m2) + k, h(j1 + j2 - j3) - k, h(j1 - m1) - k, h(j2 + m2) - k]
        if min(args) < 0:
            continue
        den = 1
        for x in args:
            den *= factorial(x)
        s += Fraction((-1) ** k, den)
    if s == 0:
        return 0.0
    phase = -1 if h(j1 - j2 - m3) % 2 else 1
    return _signed_sqrt(pre * s * s, phase * (1 if s > 0 else -1))


def make_symbols():
    import random
    w6, w3 = [], []
    r = range(0, 7)
    for j1 in r:
        for j2 in r:
            for j3 in r:
                if _delta2(j1, j2, j3) is None:
                    continue
                for l1 in r:
                    for l2 in r:
                        for l3 in r:
                            v = w6j_exact(j1, j2, j3, l1, l2, l3)
                            if v != 0.0:
                                w6.append([j1, j2, j3, l1, l2, l3, v])
    rng = random.Random(7)
    n_exhaustive = len(w6)
    while len(w6) < n_exhaustive + 600:
        j = [rng.randrange(0, 25) for _ in range(6)]
        v = w6j_exact(*j)
        if v != 0.0:
            w6.append(j + [v])
    r3 = range(0, 7)
    for j1 in r3:
        for j2 in r3:
            for j3 in r3:
                if _delta2(j1, j2, j3) is None:
                    continue
                for m1 in range(-j1, j1 + 1, 2):
                    for m2 in range(-j2, j2 + 1, 2):
                        m3 = -m1 - m2
                        v = w3j_exact(j1, j2, j3, m1, m2, m3)
                        if v != 0.0:
                            w3.append([j1, j2, j3, m1, m2, m3, v])
    with open(os.path.join(HERE, "w6j_w3j.json"), "w") as f:
        json.dump({"w6j": w6, "w3j": w3}, f, separators=(",", ":"))
    return len(w6), len(w3)


def fingerprint(sb) -> str:
    """SHA-256 over the superblock inputs: wave, operator blocks, basis tables."""
    h = hashlib.sha256()
    h.update(sb.wave.data.tobytes())
    for m in (sb.sys, sb.env):
        for s in m.ham.subs:
            h.update(s.mat.tobytes(order="F"))
        for bs in m.sub:
            for k in ("elec_up", "elec_down", "spin_sd", "spin_sz", "num_sn"):
                for s in getattr(bs, k).subs:
                    h.update(repr((s.num_up, s.num_down, s.down_dif)).encode())
                    h.update(s.mat.tobytes(order="F"))
    for bsis in (sb.sys_bs, sb.env_bs):
        for mp in bsis.maps:
            h.update(repr((mp.new_num_up, mp.new_num_down, mp.subs)).encode())
    return h.hexdigest()


GOLDEN_CASES = (("tiny", 21, 4, 8), ("small", 21, 6, 12), ("small_gc", 21, 10, 20), ("cyl4", 21, 20, 40))


def make_oracle_fixtures():
    import numpy as np
    from grand_sql_tj_b200 import synth
    from oracle import oracle
    for name, seed, kmin, kmax in GOLDEN_CASES:
        sb = synth.workload(name, seed=seed)
        out = oracle.model_wave(sb).data
        e0, iters, psi = oracle.lanczos(sb, 1e-10)
        r, blk, ev = oracle.truncation(psi, 0, kmin, kmax, 1e-12)
        np.savez_compressed(
            os.path.join(HERE, "oracle_%s.npz" % name),
            fingerprint=np.array(fingerprint(sb)), seed=seed, hpsi=out, e0=e0, iters=iters,
            trunc=np.array([r.num_state, r.trunc_err, r.entropy1, r.entropy2, r.entropys]),
            trunc_kept=np.array([kmin, kmax]), rho_eigs=ev, psi0=psi.data,
            trunc_sectors=np.array([[s.num_up, s.num_down, s.mat.shape[0], s.mat.shape[1]] for s in blk.subs]))


if __name__ == "__main__":
    print("symbols (6j, 3j):", make_symbols())
    make_oracle_fixtures()
    print("oracle fixtures:", [c[0] for c in GOLDEN_CASES])
