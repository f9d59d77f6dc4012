"""Wavefunction prediction and full sweeps, on the CPU.

  * tj_wave_trans compiles wave_trans_LR / wave_trans_RL (code/tjsq/
    dmrg_sub.f90:1093-1384) into grouped-GEMM task lists; executed with numpy
    and normalised they must equal the oracle's restatement on every call of
    a truncated run's sweeps (<= 1e-14 absolute on the normalised vector).
  * A full run of the restated schedule (warm-up, two half-sweeps, one full
    sweep; Get_Ground_State, main.f90:96-187) on the oracle with no
    truncation: every step's superblock is the whole cluster, so every
    step's energy must be the exact ground energy (tests/ed.py, <= 1e-10
    relative), and the predicted vector must already be the ground state
    (Lanczos stops after at most 3 vectors at every step but the first of a
    sweep from a random start).
"""
import numpy as np
import pytest

from grand_sql_tj_b200.lattice import Geometry
from grand_sql_tj_b200.lib import wave_trans_plan_export
from grand_sql_tj_b200.sweep import Dmrg, DmrgParams
from tests.plan_exec import execute


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


@pytest.mark.parametrize("nx,ny,ne,kept", [(6, 2, 10, 24), (3, 4, 8, 30)])
def test_wave_trans_plan_matches_oracle(product_lib, oracle_lib, nx, ny, ne, kept):
    geo = Geometry(nx, ny, t=1.0, J=1.0 / 3.0, t2=-0.2 if ny == 4 else 0.0, esite=-0.2, up_bias=1)
    be = RecordingOracle()
    d = Dmrg(geo, be, DmrgParams(n_elec=ne, kept_min=kept * 2 // 3, kept_max=kept, seed=3, lanzero=1e-8))
    n = geo.num_site
    d.warm_up()
    d.left_to_right(n // 2 - 1, n - 2, restart=False)
    d.right_to_left(n - 2, 1)
    d.left_to_right(1, n - 2)
    assert len(be.calls) > 10
    for (dr, sbs, ebs, st, et, old, ref) in be.calls:
        plan = wave_trans_plan_export(dr, sbs, ebs, st, et, old, ref.like())
        got = execute(plan, old.data)
        got = got / np.linalg.norm(got)
        assert np.max(np.abs(got - ref.data[:ref.dim])) <= 1e-14


@pytest.mark.parametrize("nx,ny,ne,t2", [(4, 2, 6, 0.0), (2, 4, 6, -0.2)])
def test_oracle_sweeps_equal_exact_diagonalisation(oracle_lib, nx, ny, ne, t2):
    from oracle.oracle import OracleBackend
    from tests import ed
    geo = Geometry(nx, ny, t=1.0, J=1.0 / 3.0, t2=t2, esite=-0.1, up_bias=1)
    e_ed = ed.ground_energy(Geometry(nx, ny, t=1.0, J=1.0 / 3.0, t2=t2, esite=-0.1, up_bias=1), ne)[0]
    d = Dmrg(geo, OracleBackend(), DmrgParams(n_elec=ne, kept_min=10 ** 5, kept_max=10 ** 6, lanzero=1e-12,
                                               lanzero_warm=1e-12, seed=3))
    recs = d.ground_state(sweeps=1)
    full = [r for r in recs if r.sys_len + r.env_len + 2 == geo.num_site]
    assert len(full) >= 3 * (geo.num_site - 3)
    for r in full:
        assert abs(r.energy - e_ed) <= 1e-10 * abs(e_ed), (r.phase, r.sys_len, r.energy, e_ed)
    starts = {"L->R0"}
    seen = set()
    for r in full:
        if r.phase in seen:
            assert r.iters <= 3, (r.phase, r.sys_len, r.iters)
        seen.add(r.phase)
    assert starts <= seen
