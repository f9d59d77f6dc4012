"""Operator renormalisation (tj_get_hamiltonian) and the DMRG it completes, on the B200.

  * every Get_Hamiltonian_Sys/Env call of a warm-up run, on the device,
    against the oracle's restatement on the same inputs (<= 1e-13 of the
    largest entry; identical sub-block records);
  * the renormalisation of the 4x24 m = 2000 system block (synthetic
    operators, random truncation operator) against the oracle (<= 1e-12);
  * a warm-up run driven entirely through the C ABI on the device (Lanczos,
    truncation, renormalisation) with every block kept whole, against exact
    diagonalisation of the full cluster (<= 1e-10 relative), as the oracle
    is held to it in test_ed_cpu.py.
"""
import os

import numpy as np
import pytest

from grand_sql_tj_b200 import synth
from grand_sql_tj_b200.lattice import Geometry
from grand_sql_tj_b200.structs import OPS
from grand_sql_tj_b200.sweep import Dmrg, DmrgParams

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx(product_lib):
    from grand_sql_tj_b200.lib import Context
    c = Context(0)
    yield c
    c.close()


def _arrays(m):
    blocks = [m.ham] + [getattr(s, k) for s in m.sub for k in OPS]
    recs = [(sb.num_up, sb.num_down, sb.down_dif, sb.mat.shape) for b in blocks for sb in b.subs]
    data = [sb.mat.reshape(-1, order="F") for b in blocks for sb in b.subs]
    return recs, (np.concatenate(data) if data else np.zeros(0))


def _same(got, ref, tol):
    rg, dg = _arrays(got)
    rr, dr = _arrays(ref)
    assert rg == rr
    assert got.len == ref.len and len(got.sub) == len(ref.sub)
    if dr.size:
        assert np.max(np.abs(dg - dr)) <= tol * np.max(np.abs(dr))


class RecordingOracle:
    def __init__(self):
        from oracle.oracle import OracleBackend
        self.o = OracleBackend()
        self.calls = []

    def __getattr__(self, k):
        return getattr(self.o, k)

    def get_hamiltonian(self, lat, side, mshift, pre, basis, trun):
        m = self.o.get_hamiltonian(lat, side, mshift, pre, basis, trun)
        self.calls.append((lat, side, mshift, pre, basis, trun, m))
        return m


@pytest.mark.parametrize("nx,ny,ne,kept,t2", [(6, 2, 10, 20, 0.0), (4, 4, 14, 40, -0.2)])
def test_renorm_matches_oracle_on_warmup(ctx, oracle_lib, nx, ny, ne, kept, t2):
    geo = Geometry(nx, ny, t=1.0, J=1.0 / 3.0, t2=t2, esite=-0.4, up_bias=1)
    be = RecordingOracle()
    Dmrg(geo, be, DmrgParams(n_elec=ne, kept_min=kept // 2, kept_max=kept, seed=3)).warm_up(lanzero=1e-10)
    for (lat, side, mshift, pre, basis, trun, ref) in be.calls:
        got = ctx.get_hamiltonian(lat, side, mshift, pre, basis, trun)
        _same(got, ref, 1e-13)


@pytest.mark.parametrize("side", [0, 1])
def test_renorm_headline_block(ctx, oracle_lib, side):
    from oracle import oracle
    oracle.set_threads(os.cpu_count() or 1)
    rc = synth.renorm_case("cyl4x24_m2000", side=side)
    ref = oracle.get_hamiltonian(rc.lat, rc.side, rc.mshift, rc.pre, rc.basis, rc.trun)
    got = ctx.get_hamiltonian(rc.lat, rc.side, rc.mshift, rc.pre, rc.basis, rc.trun)
    _same(got, ref, 1e-12)
    st = ctx.stats()
    assert st.renorm_flops > 0 and st.renorm_ms > 0


@pytest.mark.parametrize("nx,ny,ne,t2,esite", [(4, 2, 6, 0.0, -0.3), (3, 4, 10, -0.2, 0.0), (4, 2, 0, 0.0, -0.8)])
def test_device_dmrg_equals_exact_diagonalisation(ctx, nx, ny, ne, t2, esite):
    from grand_sql_tj_b200.lib import DeviceBackend
    from tests import ed
    ub = 1 if ne > 0 else 0
    geo = Geometry(nx, ny, t=1.0, J=1.0 / 3.0, t2=t2, esite=esite, up_bias=ub)
    d = Dmrg(geo, DeviceBackend(ctx), DmrgParams(n_elec=ne, kept_min=10 ** 6, kept_max=10 ** 6, seed=3))
    recs = d.warm_up(lanzero=1e-13)
    ref_geo = Geometry(nx, ny, t=1.0, J=1.0 / 3.0, t2=t2, esite=esite, up_bias=ub)
    e_ed = ed.ground_energy(ref_geo, ne)[0] if ub else ed.grand_canonical_ground_energy(ref_geo)
    assert abs(recs[-1].energy - e_ed) <= 1e-10 * abs(e_ed), (recs[-1].energy, e_ed)
