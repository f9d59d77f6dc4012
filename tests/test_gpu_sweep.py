"""Full DMRG runs through the C ABI on the B200 (Lanczos, truncation,
operator renormalisation and wavefunction prediction all on the device).

  * untruncated run of the reference's schedule (Get_Ground_State,
    main.f90:96-187): every step's energy equals exact diagonalisation
    (<= 1e-10 relative), and the carried vector is already the ground state
    (<= 3 Lanczos vectors after each sweep's first step);
  * every tj_wave_trans call of a truncated run against the oracle on the
    same inputs (<= 1e-13 absolute on the normalised vector);
  * a truncated run on the device against the same run on the oracle (same
    start vectors, same schedule): in the full sweep, energies per step
    within 1e-10 per site, the same number of kept states, truncation errors
    within 10 % (or both below 1e-13); before it (warm-up and the start
    half-sweeps), energies within 1e-7 per site, since a density matrix with
    fewer nonzero eigenvalues than kept states leaves the kept zero-weight
    states to any basis of its null space, DSYEV's and the device's differing
    (measured: 1.4e-9 per site before the sweep, 4e-12 in it).
"""
import numpy as np
import pytest

from grand_sql_tj_b200.lattice import Geometry
from grand_sql_tj_b200.sweep import Dmrg, DmrgParams

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx(product_lib):
    from grand_sql_tj_b200.lib import Context
    c = Context(0)
    yield c
    c.close()


def test_device_sweeps_equal_exact_diagonalisation(ctx):
    from grand_sql_tj_b200.lib import DeviceBackend
    from tests import ed
    geo = Geometry(6, 2, t=1.0, J=1.0 / 3.0, esite=-0.1, up_bias=1)
    e_ed = ed.ground_energy(Geometry(6, 2, t=1.0, J=1.0 / 3.0, esite=-0.1, up_bias=1), 10)[0]
    d = Dmrg(geo, DeviceBackend(ctx), DmrgParams(n_elec=10, kept_min=10 ** 5, kept_max=10 ** 6, lanzero=1e-12,
                                                  lanzero_warm=1e-12, seed=3))
    recs = d.ground_state(sweeps=1)
    full = [r for r in recs if r.sys_len + r.env_len + 2 == geo.num_site]
    assert len(full) >= 3 * (geo.num_site - 3)
    for r in full:
        assert abs(r.energy - e_ed) <= 1e-10 * abs(e_ed), (r.phase, r.sys_len, r.energy, e_ed)
    seen = set()
    for r in full:
        if r.phase in seen:
            assert r.iters <= 3, (r.phase, r.sys_len, r.iters)
        seen.add(r.phase)


class RecordingOracle:
    def __init__(self):
        from oracle.oracle import OracleBackend
        self.o = OracleBackend()
        self.calls = []

    def __getattr__(self, k):
        return getattr(self.o, k)

    def wave_trans(self, direction, sys_bs, env_bs, sys_trun, env_trun, old, new_wave):
        old_c = old.copy()
        w = self.o.wave_trans(direction, sys_bs, env_bs, sys_trun, env_trun, old, new_wave)
        self.calls.append((direction, sys_bs, env_bs, sys_trun, env_trun, old_c, w.copy()))
        return w


def test_device_wave_trans_matches_oracle(ctx, oracle_lib):
    geo = Geometry(6, 2, t=1.0, J=1.0 / 3.0, esite=-0.2, up_bias=1)
    be = RecordingOracle()
    d = Dmrg(geo, be, DmrgParams(n_elec=10, kept_min=16, kept_max=24, seed=3, lanzero=1e-8))
    d.warm_up()
    d.left_to_right(5, 10, restart=False)
    d.right_to_left(10, 1)
    assert len(be.calls) > 10
    for (dr, sbs, ebs, st, et, old, ref) in be.calls:
        got = ctx.wave_trans(dr, sbs, ebs, st, et, old, ref.like())
        assert np.max(np.abs(got.data[:got.dim] - ref.data[:ref.dim])) <= 1e-13


def test_device_run_matches_oracle_run(ctx, oracle_lib):
    """A 2x8 ladder at 14 electrons keeping 48 multiplets (both sides truncated
    from the third warm-up step on): the same schedule on the device and on
    the oracle from the same seeded start vectors."""
    from grand_sql_tj_b200.lib import DeviceBackend
    from oracle.oracle import OracleBackend
    geo = Geometry(8, 2, t=1.0, J=1.0 / 3.0, esite=0.0, up_bias=1)
    p = DmrgParams(n_elec=14, kept_min=32, kept_max=48, seed=11, lanzero=1e-10, lanzero_warm=1e-10)
    dev = Dmrg(geo, DeviceBackend(ctx), p).ground_state(sweeps=1)
    ref = Dmrg(Geometry(8, 2, t=1.0, J=1.0 / 3.0, esite=0.0, up_bias=1), OracleBackend(), p).ground_state(sweeps=1)
    assert len(dev) == len(ref)
    n = geo.num_site
    for a, b in zip(dev, ref):
        assert (a.phase, a.sys_len, a.env_len) == (b.phase, b.sys_len, b.env_len)
        if a.phase in ("warmup", "L->R0", "R->L0"):
            assert abs(a.energy - b.energy) / n <= 1e-7, (a.phase, a.sys_len, a.energy, b.energy)
            continue
        assert abs(a.energy - b.energy) / n <= 1e-10, (a.phase, a.sys_len, a.energy, b.energy)
        assert a.num_state == b.num_state or max(abs(a.trunc_err), abs(b.trunc_err)) <= 1e-14
        if max(a.trunc_err, b.trunc_err) > 1e-13:
            assert abs(a.trunc_err - b.trunc_err) <= 0.1 * max(a.trunc_err, b.trunc_err)


def test_residency_gives_the_same_run(product_lib):
    """Blocks kept on the device (tj_set_residency), written into pooled
    page-locked host buffers, give the same run as uploads from ordinary host
    arrays, bit for bit, with uploads served from the
    kept copies; a kept array that the caller changes where its fingerprint
    looks is dropped and read from the host again."""
    from grand_sql_tj_b200.lib import Context, DeviceBackend
    p = DmrgParams(n_elec=14, kept_min=32, kept_max=48, seed=11, lanzero=1e-10, lanzero_warm=1e-10)
    c0, c1 = Context(0), Context(0)
    try:
        c1.set_residency(2.0)
        c1.use_host_pool(True)
        geo = Geometry(8, 2, t=1.0, J=1.0 / 3.0, esite=0.0, up_bias=1)
        ref = Dmrg(Geometry(8, 2, t=1.0, J=1.0 / 3.0, esite=0.0, up_bias=1), DeviceBackend(c0), p).ground_state(1)
        d = Dmrg(geo, DeviceBackend(c1), p)
        got = d.ground_state(1)
        assert c1.stats().res_hits > 20 and c0.stats().res_hits == 0
        assert [r.energy for r in got] == [r.energy for r in ref]
        assert [r.trunc_err for r in got] == [r.trunc_err for r in ref]
        L = 5
        lat = geo.lattice(L, geo.num_site - L - 2)
        pre = d.sysblocks[L]
        a = c1.get_hamiltonian(lat, 0, 0, pre, d.sysbs[L + 1], d.systruns[L + 1])
        b = c0.get_hamiltonian(lat, 0, 0, pre, d.sysbs[L + 1], d.systruns[L + 1])
        assert np.array_equal(a._packed.data, b._packed.data)
        hits = c1.stats().res_hits
        pre._packed.data[0] += 1.0
        a = c1.get_hamiltonian(lat, 0, 0, pre, d.sysbs[L + 1], d.systruns[L + 1])
        b = c0.get_hamiltonian(lat, 0, 0, pre, d.sysbs[L + 1], d.systruns[L + 1])
        assert np.array_equal(a._packed.data, b._packed.data)
        # the changed model is read from the host: the one upload still served
        # from a kept copy is the truncation operator's
        assert c1.stats().res_hits == hits + 1
    finally:
        c0.close()
        c1.close()
