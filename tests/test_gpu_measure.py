"""Measurement operators on the B200 (tj_get_oper, tj_change_oper,
tj_update_trun, tj_block_mul_block_ndia) and the correlations they give.

  * every call that the restated Get_density_cor makes for <S_i . S_j>, run
    on the device and on the oracle with the same inputs, on a truncated
    2x8 ladder: identical sub-block records, entries within 1e-12 of the
    largest; the correlations within 1e-10;
  * the same for every call of the restated Get_mSCOP_Operator_Cor0 (the
    singlet pair correlation, bonds along and across the ladder);
  * every call of the restated Measurement (main.f90:191-332) on a truncated
    6x6 cylinder with t' = -0.2 (the six-leg branch of the pair correlator
    included), device against oracle on the oracle's wavefunction;
  * <S_i . S_j> from an untruncated device run on a 2x6 ladder against
    exact diagonalisation (3e-8, the convergence of the Lanczos vector).
"""
import numpy as np
import pytest

from grand_sql_tj_b200.lattice import Geometry
from grand_sql_tj_b200.measure import Chains, density_cor, measurement, pairing_cor
from grand_sql_tj_b200.sweep import Dmrg, DmrgParams, site_block_ops

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx(product_lib):
    from grand_sql_tj_b200.lib import Context
    c = Context(0)
    yield c
    c.close()


class Pair:
    """Runs each measurement call on the device and on the oracle and compares."""

    def __init__(self, dev, ora):
        self.dev, self.ora, self.calls = dev, ora, 0

    def _same(self, a, b):
        ra = [(s.num_up, s.num_down, s.down_dif, s.mat.shape) for s in a.subs]
        rb = [(s.num_up, s.num_down, s.down_dif, s.mat.shape) for s in b.subs]
        assert ra == rb
        assert (a.up_dif, a.down_dif, a.len) == (b.up_dif, b.down_dif, b.len)
        scale = max([float(np.max(np.abs(s.mat))) for s in b.subs if s.mat.size] + [1e-300])
        for x, y in zip(a.subs, b.subs):
            if y.mat.size:
                assert np.max(np.abs(x.mat - y.mat)) <= 1e-12 * scale
        self.calls += 1
        return b

    def __getattr__(self, name):
        def f(*a, **k):
            r_dev = getattr(self.dev, name)(*a, **k)
            r_ora = getattr(self.ora, name)(*a, **k)
            if name == "correlator":
                assert abs(r_dev - r_ora) <= 1e-10 * max(1.0, abs(r_ora)), (a[0], r_dev, r_ora)
                return r_ora
            return self._same(r_dev, r_ora)
        return f


def test_measurement_calls_match_oracle(ctx, oracle_lib):
    from grand_sql_tj_b200.lib import DeviceBackend
    from oracle.oracle import OracleBackend
    geo = Geometry(8, 2, t=1.0, J=1.0 / 3.0, esite=0.0, up_bias=1)
    ora = OracleBackend()
    d = Dmrg(geo, ora, DmrgParams(n_elec=14, kept_min=32, kept_max=48, seed=11, lanzero=1e-10, lanzero_warm=1e-10))
    n = geo.num_site
    d.warm_up()
    d.left_to_right(n // 2 - 1, n - 2, restart=False)
    d.right_to_left(n - 2, 1)
    d.left_to_right(1, n // 2 + 1)
    ch = Chains(d, d.wave)
    be = Pair(DeviceBackend(ctx), ora)
    ops = site_block_ops(1)
    for sid1 in (1, 2):
        density_cor(be, ch, d.wave, ops["st_sd"], ops["st_sd"], "B", sid1, 2, n)
    density_cor(be, ch, d.wave, ops["elec_up"], ops["elec_down"], "F", 1, 2, n)
    assert be.calls > 20
    geo.setup(d.wave.sys_len - 1, d.wave.env_len - 1)
    before = be.calls
    for ij in (1, 3):
        res = pairing_cor(be, ch, d.wave, ops, lambda i, k: int(geo.neib[i, k]), 1, 3, ij, 2, n)
        assert len(res) >= 3
    assert be.calls > before + 30


def test_device_spin_correlation_equals_ed(ctx):
    from grand_sql_tj_b200.lib import DeviceBackend
    from tests import ed
    geo = Geometry(6, 2, t=1.0, J=1.0 / 3.0, esite=0.0, up_bias=1)
    be = DeviceBackend(ctx)
    d = Dmrg(geo, be, DmrgParams(n_elec=10, kept_min=10 ** 5, kept_max=10 ** 6, lanzero=1e-14, lanzero_warm=1e-14,
                                 seed=3))
    n = geo.num_site
    d.warm_up()
    d.left_to_right(n // 2 - 1, n - 2, restart=False)
    d.right_to_left(n - 2, 1)
    d.left_to_right(1, n // 2 + 1)
    e0, psi, cl = ed.ground_energy(Geometry(6, 2, t=1.0, J=1.0 / 3.0, up_bias=1), 10)
    ops = site_block_ops(1)
    res = density_cor(be, Chains(d, d.wave), d.wave, ops["st_sd"], ops["st_sd"], "B", 1, 2, n)
    for (i, j), v in res.items():
        assert abs(v - ed.spin_correlation(cl, psi, i - 1, j - 1)) <= 3e-8, (i, j, v)


def test_six_leg_measurement_matches_oracle(ctx, oracle_lib):
    from grand_sql_tj_b200.lib import DeviceBackend
    from oracle.oracle import OracleBackend
    ora = OracleBackend()
    geo = Geometry(6, 6, t=1.0, J=1.0 / 3.0, t2=-0.2, esite=0.0, up_bias=1)
    d = Dmrg(geo, ora, DmrgParams(n_elec=32, kept_min=48, kept_max=64, lanzero=1e-8, lanzero_warm=1e-6, seed=5))
    d.ground_state(1, final_half=True)
    be = Pair(DeviceBackend(ctx), ora)
    res = measurement(be, d)
    assert any(k[0] == 5 for k in res["pair_y"])   # the six-leg branch (reference bond at site 1 + 4)
    assert all(len(v) >= 5 for v in res.values())
    assert be.calls > 60
