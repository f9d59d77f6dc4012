"""Correlation functions on the oracle against exact diagonalisation (CPU).

An untruncated run (every block kept whole) of the restated schedule on a
2x6 ladder leaves the wavefunction of the full cluster; the restated
measurement driver (grand_sql_tj_b200.measure: Get_density_cor with
Get_sys2b, measure.f90:2785-3223) then gives <S_i . S_j> and <n_i n_j> for
the pairs of both block interiors, the centre sites and across the blocks,
through the oracle's Get/Change_*_oper_*, update_trun, block_mul_block_ndia
and contraction kernels.  They must equal the exact values of tests/ed.py.
Tolerance 3e-8 absolute: the Lanczos vector is converged on its Ritz value
(1e-14), which leaves the vector itself accurate to about 1e-7.
"""
import pytest

from grand_sql_tj_b200.lattice import Geometry
from grand_sql_tj_b200.measure import Chains, density_cor
from grand_sql_tj_b200.sweep import Dmrg, DmrgParams, site_block_ops


@pytest.fixture(scope="module")
def run(oracle_lib):
    from oracle.oracle import OracleBackend
    from tests import ed
    geo = Geometry(6, 2, t=1.0, J=1.0 / 3.0, esite=0.0, up_bias=1)
    be = OracleBackend()
    d = Dmrg(geo, be, DmrgParams(n_elec=10, kept_min=10 ** 5, kept_max=10 ** 6, lanzero=1e-14,
                                  lanzero_warm=1e-14, seed=3))
    n = geo.num_site
    d.warm_up()
    d.left_to_right(n // 2 - 1, n - 2, restart=False)
    d.right_to_left(n - 2, 1)
    d.left_to_right(1, n // 2 + 1)
    e0, psi, cl = ed.ground_energy(Geometry(6, 2, t=1.0, J=1.0 / 3.0, up_bias=1), 10)
    return be, d, Chains(d, d.wave), psi, cl


@pytest.mark.parametrize("sid1", [1, 2, 3])
def test_spin_correlation_equals_ed(run, sid1):
    from tests import ed
    be, d, ch, psi, cl = run
    ops = site_block_ops(1)
    res = density_cor(be, ch, d.wave, ops["st_sd"], ops["st_sd"], "B", sid1, 2, d.N)
    assert len(res) >= 4
    for (i, j), v in res.items():
        assert abs(v - ed.spin_correlation(cl, psi, i - 1, j - 1)) <= 3e-8, (i, j, v)


def test_density_correlation_equals_ed(run):
    from tests import ed
    be, d, ch, psi, cl = run
    ops = site_block_ops(1)
    res = density_cor(be, ch, d.wave, ops["num_elec"], ops["num_elec"], "B", 2, 2, d.N)
    for (i, j), v in res.items():
        assert abs(v - ed.density_correlation(cl, psi, i - 1, j - 1)) <= 3e-8, (i, j, v)
