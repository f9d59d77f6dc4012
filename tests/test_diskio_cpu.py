"""The reference's checkpoint files (code/tjsq/block.f90:2760-3097), on the CPU.

The library's writers must produce, byte for byte, what a Fortran runtime
writes for the reference's WRITE statements -- checked against an
independent writer here (struct.pack; one record per WRITE, framed by its
4-byte length) -- and its readers must return what was written, including
records split into subrecords (negative length markers), which the Fortran
runtimes use above 2 GiB and which are made small here.  The basis text must
follow the reference's FORMAT descriptors (A4,I6 / A11,I4 / A13,I4 /
A10,I4,2X,A12,I4).  Inputs: blocks, truncations, bases and the wavefunction
of a truncated warm-up run (oracle).
"""
import struct

import numpy as np
import pytest

from grand_sql_tj_b200 import lib as L
from grand_sql_tj_b200.lattice import Geometry
from grand_sql_tj_b200.structs import OPS
from grand_sql_tj_b200.sweep import Dmrg, DmrgParams


def rec(payload: bytes, split=None) -> bytes:
    if split is None or len(payload) <= split:
        return struct.pack("<i", len(payload)) + payload + struct.pack("<i", len(payload))
    parts = [payload[i:i + split] for i in range(0, len(payload), split)]
    out = b""
    for k, p in enumerate(parts):
        lead = len(p) if k == len(parts) - 1 else -len(p)
        tail = len(p) if k == 0 else -len(p)
        out += struct.pack("<i", lead) + p + struct.pack("<i", tail)
    return out


def ints(*v):
    return struct.pack("<%di" % len(v), *v)


def block_bytes(b, split=None):
    out = rec(ints(b.len)) + rec(ints(len(b.subs))) + rec(ints(b.dim)) + rec(ints(b.up_dif)) + rec(ints(b.down_dif))
    for s in b.subs:
        r, c = s.mat.shape
        out += rec(b"") + rec(ints(s.num_up, s.num_down, s.down_dif)) + rec(ints(r, c))
        out += rec(np.asarray(s.mat, dtype="<f8").tobytes(order="F"), split)
    return out


def wave_bytes(w, split=None):
    out = rec(ints(w.sys_len)) + rec(ints(w.env_len)) + rec(ints(len(w.sectors))) + rec(ints(w.dim))
    for i, s in enumerate(w.sectors):
        out += rec(b"") + rec(ints(s.sys_num_up, s.sys_num_down)) + rec(ints(s.env_num_up, s.env_num_down))
        out += rec(ints(s.sys_dim, s.env_dim)) + rec(w.sector(i).astype("<f8").tobytes(order="F"), split)
    return out


def basis_text(b):
    lines = ["len=%6d" % b.len, "num=%6d" % len(b.maps), "dim=%6d" % b.dim]
    for m in b.maps:
        lines += ["", "idx=%6d" % 0, "num=%6d" % len(m.subs), "dim=%6d" % m.dim,
                  "new_num_up=%4d" % m.new_num_up, "new_num_down=%4d" % m.new_num_down]
        for (spos, sdim, bu, bd, su, sd) in m.subs:
            lines += ["pos=%6d" % spos, "dim=%6d" % sdim, "bl_num_up=%4d  bl_num_down=%4d" % (bu, bd),
                      "st_num_up=%4d  st_num_down=%4d" % (su, sd)]
    return "\n".join(lines) + "\n"


@pytest.fixture(scope="module")
def run(oracle_lib, product_lib):
    from oracle.oracle import OracleBackend
    geo = Geometry(6, 2, t=1.0, J=1.0 / 3.0, esite=-0.2, up_bias=1)
    d = Dmrg(geo, OracleBackend(), DmrgParams(n_elec=10, kept_min=16, kept_max=24, seed=3, lanzero=1e-8))
    d.warm_up()
    return d


def test_disk_names():
    assert L.disk_name(0, 12) == "sysblocks12"
    assert L.disk_name(4, 3) == "envtruns3"
    assert L.disk_name(6, 1) == "eigvec1"


def test_wave_bytes_and_round_trip(run, tmp_path):
    w = run.wave
    p = str(tmp_path / "eigvec1")
    L.wave_to_disk(p, w)
    assert open(p, "rb").read() == wave_bytes(w)
    back = L.wave_from_disk(p)
    assert (back.sys_len, back.env_len, back.dim) == (w.sys_len, w.env_len, w.dim)
    assert [vars(a) for a in back.sectors] == [vars(b) for b in w.sectors]
    assert np.array_equal(back.data[:back.dim], w.data[:w.dim])
    q = str(tmp_path / "split")
    open(q, "wb").write(wave_bytes(w, split=40))      # subrecords of 40 bytes
    assert np.array_equal(L.wave_from_disk(q).data[:w.dim], w.data[:w.dim])


def test_block_and_model_round_trip(run, tmp_path):
    m = run.sysblocks[max(run.sysblocks)]
    t = run.systruns[max(run.systruns)]
    p = str(tmp_path / "systruns5")
    L.block_to_disk(p, t)
    assert open(p, "rb").read() == block_bytes(t)
    b = L.block_from_disk(p)
    assert [(s.num_up, s.num_down, s.down_dif) for s in b.subs] == [(s.num_up, s.num_down, s.down_dif) for s in t.subs]
    for x, y in zip(b.subs, t.subs):
        assert np.array_equal(x.mat, y.mat)
    q = str(tmp_path / "sysblocks5")
    L.model_to_disk(q, m)
    want = rec(ints(m.len)) + block_bytes(m.ham)
    for s in m.sub:
        for k in ("elec_up", "elec_down", "spin_sd", "num_sn"):
            want += block_bytes(getattr(s, k))
    assert open(q, "rb").read() == want
    back = L.model_from_disk(q)
    assert back.len == m.len and len(back.sub) == len(m.sub)
    for a, b_ in zip([back.ham] + [getattr(s, k) for s in back.sub for k in OPS if k != "spin_sz"],
                     [m.ham] + [getattr(s, k) for s in m.sub for k in OPS if k != "spin_sz"]):
        assert len(a.subs) == len(b_.subs)
        for x, y in zip(a.subs, b_.subs):
            assert (x.num_up, x.num_down, x.down_dif) == (y.num_up, y.num_down, y.down_dif)
            assert np.array_equal(x.mat, y.mat)
    r = str(tmp_path / "split")
    open(r, "wb").write(rec(ints(m.len)) + block_bytes(m.ham, split=24) +
                        b"".join(block_bytes(getattr(s, k), split=24) for s in m.sub
                                 for k in ("elec_up", "elec_down", "spin_sd", "num_sn")))
    assert np.array_equal(L.model_from_disk(r).ham.subs[0].mat, m.ham.subs[0].mat)


def test_basis_text_and_round_trip(run, tmp_path):
    b = run.sysbs[max(run.sysbs)]
    p = str(tmp_path / "sysbs5")
    L.basis_to_disk(p, b)
    assert open(p).read() == basis_text(b)
    back = L.basis_from_disk(p)
    assert back.len == b.len and [(m.new_num_up, m.new_num_down, m.subs) for m in back.maps] == \
        [(m.new_num_up, m.new_num_down, m.subs) for m in b.maps]


def test_malformed_files_are_rejected(tmp_path):
    p = str(tmp_path / "bad")
    open(p, "wb").write(struct.pack("<i", 4) + ints(3) + struct.pack("<i", 8))   # markers disagree
    with pytest.raises(L.TjError):
        L.block_from_disk(p)
    open(p, "wb").write(rec(ints(3)))                                           # ends early
    with pytest.raises(L.TjError):
        L.wave_from_disk(p)
