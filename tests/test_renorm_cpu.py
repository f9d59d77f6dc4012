"""The operator-renormalisation compiler against the oracle, on the CPU.

tj_get_hamiltonian compiles Get_Hamiltonian_Sys/Env (code/tjsq/get_sys.f90:
4-480) into grouped-GEMM task lists without forming the enlarged operators;
here the exported lists are executed with numpy (tests/plan_exec.py) and
compared with the oracle's restatement, which builds every enlarged
operator densely and truncates it with the reference's DGEMM pairs
(update_trun_dia/ndia, code/tjsq/block.f90:1311-1503).  Inputs: every
renormalisation of a warm-up run (untruncated and truncated steps, both
sides), and synthetic blocks with random truncation operators.
Tolerance: 1e-13 of the largest entry (FP64 sums in another order); the
result's sub-block records must be identical.
"""
import numpy as np
import pytest

from grand_sql_tj_b200 import synth
from grand_sql_tj_b200.lattice import Geometry
from grand_sql_tj_b200.lib import renorm_plan_export
from grand_sql_tj_b200.structs import OPS
from grand_sql_tj_b200.sweep import Dmrg, DmrgParams
from tests.plan_exec import execute


def model_arrays(m):
    blocks = [m.ham] + [getattr(s, k) for s in m.sub for k in OPS]
    recs = [(sb.num_up, sb.num_down, sb.down_dif, sb.mat.shape) for b in blocks for sb in b.subs]
    data = [sb.mat.reshape(-1, order="F") for b in blocks for sb in b.subs]
    return recs, (np.concatenate(data) if data else np.zeros(0))


def check_plan(lat, side, mshift, pre, basis, trun, ref_model):
    plan = renorm_plan_export(lat, side, mshift, pre, basis, trun)
    got = execute(plan, plan["trun"])
    recs, ref = model_arrays(ref_model)
    res = plan["res"]
    assert res.len == ref_model.len and res.nsub == len(ref_model.sub)
    precs = [(res.subs[i].num_up, res.subs[i].num_down, res.subs[i].down_dif, (res.subs[i].row_dim, res.subs[i].sdim))
             for i in range(res.n_subs)]
    assert precs == recs
    assert res.data_len == ref.size
    if ref.size:
        assert np.max(np.abs(got - ref)) <= 1e-13 * max(np.max(np.abs(ref)), 1e-300)


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


@pytest.mark.parametrize("nx,ny,ne,kept,t2", [(4, 2, 6, 10 ** 6, 0.0), (6, 2, 10, 20, 0.0), (4, 4, 14, 40, -0.2)])
def test_renorm_plan_matches_oracle_on_warmup(product_lib, oracle_lib, nx, ny, ne, kept, t2):
    geo = Geometry(nx, ny, t=1.0, J=1.0 / 3.0, t2=t2, esite=-0.4, up_bias=1)
    be = RecordingOracle()
    Dmrg(geo, be, DmrgParams(n_elec=ne, kept_min=kept // 2, kept_max=kept, seed=3)).warm_up(lanzero=1e-10)
    assert be.calls
    for c in be.calls:
        check_plan(*c)


@pytest.mark.parametrize("name,side", [("tiny", 0), ("small", 1), ("small_gc", 0), ("cyl4", 0), ("cyl4", 1)])
def test_renorm_plan_matches_oracle_synthetic(product_lib, oracle_lib, name, side):
    from oracle import oracle
    rc = synth.renorm_case(name, side=side, seed=5)
    ref = oracle.get_hamiltonian(rc.lat, rc.side, rc.mshift, rc.pre, rc.basis, rc.trun)
    check_plan(rc.lat, rc.side, rc.mshift, rc.pre, rc.basis, rc.trun, ref)


def test_renorm_rejects_mismatched_trun(product_lib):
    from grand_sql_tj_b200.lib import TjError
    rc = synth.renorm_case("tiny", seed=2)
    bad = synth.random_trun(rc.basis, 4, np.random.default_rng(0))
    bad.subs[0].mat = np.asfortranarray(np.vstack([bad.subs[0].mat, np.zeros((1, bad.subs[0].mat.shape[1]))]))
    with pytest.raises(TjError):
        renorm_plan_export(rc.lat, rc.side, rc.mshift, rc.pre, rc.basis, bad)
