"""The C ABI of include/tj_b200.h, checked without a GPU.

libtjb200.so loads and exports every function the header declares, and each
ctypes mirror (grand_sql_tj_b200/structs.py, lib.py) has the size and field
offsets that a C compiler gives the header's struct (a small program built
with gcc against the header prints them).
"""
import ctypes as C
import os
import re
import subprocess

import pytest

from grand_sql_tj_b200 import lib as L
from grand_sql_tj_b200 import structs as S

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "tj_b200.h")

MIRRORS = {
    "tj_block_sub": S.TjBlockSub, "tj_block": S.TjBlock, "tj_block_set": S.TjBlockSet, "tj_model": S.TjModel,
    "tj_basis_sub": S.TjBasisSub, "tj_basis_map": S.TjBasisMap, "tj_basis": S.TjBasis,
    "tj_wave_sub": S.TjWaveSub, "tj_wave": S.TjWave, "tj_lattice": S.TjLattice,
    "tj_trunc_result": S.TjTruncResult, "tj_hpsi_stats": S.TjHpsiStats, "tj_tune_result": S.TjTuneResult,
    "tj_gg_cell": S.TjGgCell, "tj_gg_term": S.TjGgTerm,
    "tj_plan_operand": L.PlanOperand, "tj_plan_task": L.PlanTask, "tj_plan_cell": L.PlanCell,
    "tj_plan_upload": L.PlanUpload, "tj_plan_merge": L.PlanMerge, "tj_plan_item": L.PlanItem,
    "tj_plan_reduce": L.PlanReduce, "tj_plan_export": L.PlanExport,
    "tj_oz_job": L.OzJobC, "tj_oz_seg": L.OzSegC, "tj_oz_fam": L.OzFamC,
    "tj_oz_item": L.OzItemC, "tj_oz_cell": L.OzCellC, "tj_ozaki_export": L.OzExport,
}


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", " ", text, flags=re.S)
    return sorted(set(re.findall(r"^\s*(?:const\s+)?[A-Za-z_][A-Za-z0-9_]*\s*\**\s*(tj_[a-z0-9_]+)\s*\(",
                                 text, flags=re.M)))


def test_header_declares_the_hot_path():
    names = declared_functions()
    for must in ("tj_model_wave", "tj_lanczos_memo_new", "tj_truncation", "tj_model_wave_noalloc",
                 "tj_sys_site_env_site_cor_ndia", "tj_host_register", "tj_autotune", "tj_grouped_gemm_bench"):
        assert must in names


def test_library_exports_every_declared_function():
    lib = C.CDLL(L.LIB_PATH)
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing


def test_struct_layouts_match_the_header(tmp_path):
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "tj_b200.h"', "int main(void) {"]
    for cname, cls in MIRRORS.items():
        lines.append('printf("%s size %%zu\\n", sizeof(%s));' % (cname, cname))
        for f in cls._fields_:
            lines.append('printf("%s %s %%zu\\n", offsetof(%s, %s));' % (cname, f[0], cname, f[0]))
    lines.append("return 0; }")
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "layout"
    cc = subprocess.run(["gcc", "-std=c11", "-I", os.path.dirname(HEADER), str(src), "-o", str(exe)],
                        capture_output=True, text=True)
    if cc.returncode != 0:
        pytest.fail(cc.stderr[-2000:])
    got = {}
    for line in subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.splitlines():
        a, b, v = line.split()
        got[(a, b)] = int(v)
    for cname, cls in MIRRORS.items():
        assert got[(cname, "size")] == C.sizeof(cls), cname
        for f in cls._fields_:
            assert got[(cname, f[0])] == getattr(cls, f[0]).offset, (cname, f[0])


def test_host_pool_size_classes():
    """HostPool rounds sizes up to eight classes per octave (at most 1/8 more)."""
    from grand_sql_tj_b200.lib import HostPool
    prev = 0
    for n in list(range(1, 70000, 97)) + [10 ** 6, 3 * 10 ** 6 + 7, 2 ** 24, 2 ** 24 + 1]:
        c = HostPool.size_class(n)
        assert c >= n and c >= 4096 and c <= max(4096, n + n // 8 + 1)
        assert c >= prev
        prev = c
