"""Correlation functions on the oracle against exact diagonalisation (CPU).

An untruncated run (every block kept whole) of the restated schedule on a
2x6 ladder leaves the wavefunction of the full cluster; the restated
measurement driver (grand_sql_tj_b200.measure: Get_density_cor with
Get_sys2b, measure.f90:2785-3223) then gives <S_i . S_j> and <n_i n_j> for
the pairs of both block interiors, the centre sites and across the blocks,
through the oracle's Get/Change_*_oper_*, update_trun, block_mul_block_ndia
and contraction kernels.  They must equal the exact values of tests/ed.py.
The singlet pair correlation <D+_(i,j) D_(k,l)> of the restated
Get_mSCOP_Operator_Cor0 (measure.f90:3377-3507) is checked the same way, on
the ladder (pairs in the system block and across the blocks) and on a
6-leg cylinder of two columns (the branch the reference takes for ny >= 6).
Finally the restated Measurement (main.f90:191-332) gives all five families (spin, density, single-particle
sum_s <c+_is c_js>, pairs along y and x) equal to exact diagonalisation.
Tolerance 3e-8 absolute: the Lanczos vector is converged on its Ritz value
(1e-14), which leaves the vector itself accurate to about 1e-7.
"""
import pytest

from grand_sql_tj_b200.lattice import Geometry
from grand_sql_tj_b200.measure import Chains, density_cor, measurement, pairing_cor
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


def _neib(geo, wave):
    geo.setup(wave.sys_len - 1, wave.env_len - 1)
    return lambda i, k: int(geo.neib[i, k])


def _check_pairs(res, neib, ij, cl, psi):
    from tests import ed
    for (s1, s3, j), v in res.items():
        ref = ed.singlet_pair_correlation(cl, psi, s1 - 1, neib(s1, ij) - 1, s3 - 1, neib(s3, j) - 1)
        assert abs(v - ref) <= 3e-8, (s1, s3, j, v, ref)


@pytest.mark.parametrize("ij", [1, 3])
def test_pairing_correlation_equals_ed(run, ij):
    be, d, ch, psi, cl = run
    neib = _neib(d.geo, d.wave)
    res = pairing_cor(be, ch, d.wave, site_block_ops(1), neib, 1, 1, ij, 2, d.N)
    assert len(res) >= (6 if ij == 1 else 3)
    _check_pairs(res, neib, ij, cl, psi)


def test_pairing_six_leg_branch_equals_ed(oracle_lib):
    from oracle.oracle import OracleBackend
    from tests import ed
    geo = Geometry(2, 6, t=1.0, J=1.0 / 3.0, esite=0.0, up_bias=1)
    be = OracleBackend()
    d = Dmrg(geo, be, DmrgParams(n_elec=10, kept_min=10 ** 5, kept_max=10 ** 6, lanzero=1e-14,
                                  lanzero_warm=1e-14, seed=3))
    n = geo.num_site
    d.warm_up()
    d.left_to_right(n // 2 - 1, n - 2, restart=False)
    d.right_to_left(n - 2, 1)
    d.left_to_right(1, n // 2 + 1)
    e0, psi, cl = ed.ground_energy(Geometry(2, 6, t=1.0, J=1.0 / 3.0, up_bias=1), 10)
    neib = _neib(geo, d.wave)
    res = pairing_cor(be, Chains(d, d.wave), d.wave, site_block_ops(1), neib, 1, 1, 1, 6, n)
    assert (5, 11, 1) in res
    _check_pairs(res, neib, 1, cl, psi)


def test_measurement_driver_equals_ed(run):
    from tests import ed
    be, d, ch, psi, cl = run
    m = measurement(be, d)
    exact = {"spin": ed.spin_correlation, "density": ed.density_correlation, "elec": ed.hopping_correlation}
    for name, f in exact.items():
        assert len(m[name]) >= 5
        for (i, j), v in m[name].items():
            assert abs(v - f(cl, psi, i - 1, j - 1)) <= 3e-8, (name, i, j, v)
    neib = _neib(d.geo, d.wave)
    _check_pairs(m["pair_y"], neib, 1, cl, psi)
    _check_pairs(m["pair_x"], neib, 3, cl, psi)
    assert len(m["pair_y"]) >= 6 and len(m["pair_x"]) >= 3
