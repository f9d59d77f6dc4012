"""Correlator contractions (measure.f90) compiled by the product, executed with
numpy on the CPU, against the oracle's restatement of the same routines."""
import numpy as np
import pytest

from grand_sql_tj_b200 import synth
from grand_sql_tj_b200.lib import cor_plan_export
from grand_sql_tj_b200.structs import block_transfer_trans
from tests.plan_exec import execute


def cases(sb, site):
    s0, e0 = sb.sys.sub[0], sb.env.sub[0]
    eu, sd = site(0), site(3)
    return [
        ("measure_sys_block", s0.num_sn, None, "B"),
        ("measure_env_block", e0.num_sn, None, "B"),
        ("sys_block_env_block_cor_dia", s0.num_sn, e0.num_sn, "B"),
        ("sys_block_env_block_cor_ndia", s0.spin_sd, block_transfer_trans(e0.spin_sd), "B"),
        ("sys_block_env_block_cor_ndia", s0.elec_up, block_transfer_trans(e0.elec_down), "F"),
        ("sys_block_site_cor_ndia", s0.elec_up, eu, "F"),
        ("sys_block_site_cor_ndia", s0.spin_sd, sd, "B"),
        ("env_block_site_cor_ndia", e0.elec_up, eu, "F"),
        ("env_block_site_cor_ndia", e0.spin_sd, sd, "B"),
        ("sys_block_env_site_cor_ndia", s0.elec_up, eu, "F"),
        ("sys_block_env_site_cor_ndia", s0.spin_sd, sd, "B"),
        ("sys_site_env_block_cor_ndia", eu, block_transfer_trans(e0.elec_down), "F"),
        ("sys_site_env_block_cor_ndia", sd, block_transfer_trans(e0.spin_sd), "B"),
        ("sys_site_env_site_cor_ndia", eu, eu, "F"),
        ("sys_site_env_site_cor_ndia", sd, sd, "B"),
    ]


@pytest.mark.parametrize("wl", ["small", "small_gc", "cyl4"])
def test_correlators_match_oracle(wl, product_lib, oracle_lib):
    from oracle import oracle
    sb = synth.workload(wl, seed=8)
    ub = sb.lat.up_bias
    site = lambda k: oracle.site_operator(k, ub)
    for name, a, b, flag in cases(sb, site):
        ref = oracle.correlator(name, a, b, sb.sys_bs, sb.env_bs, sb.wave, flag)
        plan = cor_plan_export(name, a, b, sb.sys_bs, sb.env_bs, sb.wave, flag)
        out = execute(plan, sb.wave.data)
        got = float(out @ sb.wave.data)
        assert abs(got - ref) <= 1e-12 * max(1.0, abs(ref)), (name, flag, got, ref)
