"""The oracle pinned to exact diagonalisation (CPU).

The oracle restates the reference's Fortran; to show that the restatement
computes the t-J model the reference states (code/tjsq/common.f90:1-4), a
warm-up run (dmrg_sub.f90:553-727 restated by grand_sql_tj_b200.sweep) with
no truncation -- every enlarged block kept whole -- must give the exact
ground energy of the full cluster.  That run goes through every oracle
routine of the path: model_wave with hmerge and its 14 term kernels,
lanczos_memo_new, and Get_Hamiltonian_Sys/Env with the block updates and
update_trun (here with unit truncation matrices, as the reference's
warm-up uses them).  The exact energy comes from tests/ed.py, which builds
the Hamiltonian in the Fock space with no code shared with the oracle.

Tolerance: |E_DMRG - E_ED| <= 1e-10 |E_ED| (Lanczos to 1e-13 on the Ritz
value; both in FP64).
"""
import pytest

from grand_sql_tj_b200.lattice import Geometry
from grand_sql_tj_b200.sweep import Dmrg, DmrgParams

# nx, ny, electrons (canonical, up_bias = 1; 0 = grand-canonical), t', esite
CASES = [
    (4, 2, 6, 0.0, 0.0),      # 2x4 ladder, 2 holes
    (4, 2, 6, 0.0, -0.3),     # with a chemical potential
    (6, 2, 10, 0.0, 0.0),     # 2x6 ladder
    (3, 4, 10, 0.0, 0.0),     # 4-leg cylinder (periodic in y), 3 columns
    (3, 4, 10, -0.2, 0.0),    # with next-nearest-neighbour hopping t' = -0.2 (J2 = J t'^2)
    (3, 4, 10, 0.3, 0.0),     # t' of the other sign
    (4, 2, 0, 0.0, -0.8),     # grand-canonical labels (the shipped up_bias = 0 mode)
]


@pytest.mark.parametrize("nx,ny,ne,t2,esite", CASES)
def test_oracle_dmrg_equals_exact_diagonalisation(oracle_lib, nx, ny, ne, t2, esite):
    from oracle.oracle import OracleBackend
    from tests import ed
    ub = 1 if ne > 0 else 0
    geo = Geometry(nx, ny, t=1.0, J=1.0 / 3.0, t2=t2, esite=esite, up_bias=ub)
    d = Dmrg(geo, OracleBackend(), DmrgParams(n_elec=ne, kept_min=10 ** 6, kept_max=10 ** 6, seed=3))
    recs = d.warm_up(lanzero=1e-13)
    assert recs[-1].sys_len + recs[-1].env_len + 2 == geo.num_site
    ref_geo = Geometry(nx, ny, t=1.0, J=1.0 / 3.0, t2=t2, esite=esite, up_bias=ub)
    e_ed = ed.ground_energy(ref_geo, ne)[0] if ub else ed.grand_canonical_ground_energy(ref_geo)
    assert abs(recs[-1].energy - e_ed) <= 1e-10 * abs(e_ed), (recs[-1].energy, e_ed)


def test_ed_helper_two_site_values():
    """The ED helper on hand-checkable cases: one hole hopping on a 2-site bond
    (E = -t) and two spins (E = -J: J (S.S - 1/4) at S = 0)."""
    import numpy as np
    from tests.ed import TJCluster
    bonds = [(0, 1, 1.0, 1.0 / 3.0)]
    for n_el, e0 in ((2, -1.0 / 3.0),):
        cl = TJCluster(2, bonds, np.zeros(2), n_el)
        w = np.linalg.eigvalsh(cl.hamiltonian().toarray())
        assert abs(w[0] - e0) < 1e-14
    # 3 sites in a line, 2 electrons: the singlet ground state lies below -J
    cl = TJCluster(3, [(0, 1, 1.0, 1.0 / 3.0), (1, 2, 1.0, 1.0 / 3.0)], np.zeros(3), 2)
    H = cl.hamiltonian().toarray()
    assert np.allclose(H, H.T)
    assert np.linalg.eigvalsh(H)[0] < -1.0 / 3.0


def test_ed_pair_operator_known_answers():
    """The ED singlet pair operator on two sites with two electrons: the
    ground state of J > 0 is the singlet, <D+ D> = 1; the Sz = 0 triplet
    gives 0."""
    import numpy as np
    from tests import ed
    cl = ed.TJCluster(2, [(0, 1, 0.0, 1.0)], np.zeros(2), 2)
    w, v = np.linalg.eigh(cl.hamiltonian().toarray())
    assert abs(ed.singlet_pair_correlation(cl, v[:, 0], 0, 1, 0, 1) - 1.0) <= 1e-14
    assert abs(ed.singlet_pair_correlation(cl, v[:, 1], 0, 1, 0, 1)) <= 1e-14
    # D_(i,j) = D_(j,i) for the singlet
    assert abs(ed.singlet_pair_correlation(cl, v[:, 0], 0, 1, 1, 0) - 1.0) <= 1e-14
