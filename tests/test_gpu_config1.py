"""The plain method on the device: the 2x16 t-J ladder (4 holes, S = 0) kept
at m = 256 multiplets through 10 full sweeps at Lanczos tolerance 1e-10, the
reference's schedule (Get_Ground_State, main.f90:96-187) with every step --
Lanczos, truncation, operator renormalisation, wavefunction prediction -- and
the correlators of Measurement (main.f90:191-332) on the B200, against the
oracle's run of the same schedule from the same seed
(tests/golden/config1_ladder16_m256.json, made by make_config1.py):

  * from the third full sweep on, every step's energy within 1e-10 per site,
    the same kept multiplets (unless the discarded weight is rounding noise,
    where the keep rule's comparison with trun_err = 1e-18 goes either way)
    and the truncation error within 10 % (measured: <= 7e-12 per site, 7e-4
    relative);
  * before that, energies within 1e-4 per site: while a block's density
    matrix has fewer nonzero eigenvalues than the states kept (the warm-up
    and the first sweeps), the kept zero-weight states are any basis of the
    null space -- DSYEV's (oracle, as the reference) and the device's differ,
    both valid -- and the next steps' variational spaces differ with them
    until the sweeps converge both runs to the same state (measured: 2e-5 per
    site in the warm-up, 3e-8 in the second sweep);
  * the spin, density, single-particle and singlet pair correlators of the
    converged state within 1e-6 (measured: <= 6e-10).
"""
import json
import os

import pytest

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))


@pytest.fixture(scope="module")
def device_run(product_lib):
    from grand_sql_tj_b200.lib import Context, DeviceBackend
    from tests.golden.make_config1 import config1_run
    c = Context(0)
    try:
        d, cors = config1_run(DeviceBackend(c))
    finally:
        c.close()
    with open(os.path.join(HERE, "golden", "config1_ladder16_m256.json")) as f:
        ref = json.load(f)
    return d, cors, ref


EARLY = ("warmup", "L->R0", "R->L0", "L->R1", "R->L1", "L->R2", "R->L2")


def test_config1_steps_match_oracle(device_run):
    d, cors, ref = device_run
    n = d.N
    assert len(d.records) == len(ref["steps"])
    for r, (phase, sl, el, e, it, ns, te) in zip(d.records, ref["steps"]):
        assert (r.phase, r.sys_len, r.env_len) == (phase, sl, el)
        if phase in EARLY:
            assert abs(r.energy - e) / n <= 1e-4, (phase, sl, r.energy, e)
            continue
        assert abs(r.energy - e) / n <= 1e-10, (phase, sl, r.energy, e)
        # the keep rule compares the discarded weight with trun_err = 1e-18:
        # where the density matrix has no weight beyond the kept states that
        # comparison is decided by rounding (in the reference as well)
        assert r.num_state == ns or max(abs(r.trunc_err), abs(te)) <= 1e-14, (phase, sl, r.num_state, ns)
        if max(abs(r.trunc_err), abs(te)) > 1e-13:
            assert abs(r.trunc_err - te) <= 0.1 * max(abs(r.trunc_err), abs(te)), (phase, sl, r.trunc_err, te)


def test_config1_correlators_match_oracle(device_run):
    d, cors, ref = device_run
    for name, rows in ref["correlators"].items():
        got = cors[name]
        assert len(got) == len(rows), name
        for *key, v in rows:
            assert abs(got[tuple(key)] - v) <= 1e-6, (name, key, got[tuple(key)], v)
