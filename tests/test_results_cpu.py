"""Blocks and models the library writes, on the CPU (through the oracle's
entry points, which return them the same way as the device library): their
sub-blocks are views into the result array, they pack to that array without
a copy while the views stand, and a replaced sub-block makes pack() copy.
A model's operator sets are built when first read."""
import numpy as np

from grand_sql_tj_b200 import synth
from grand_sql_tj_b200.structs import OPS, PackedBlock, PackedModel


def test_truncation_block_packs_to_its_result(oracle_lib):
    from oracle import oracle
    sb = synth.workload("small")
    _, blk, _ = oracle.truncation(sb.wave, 0, 8, 16, 1e-12)
    pk = blk.pack()
    assert pk is blk._packed and not isinstance(pk, PackedBlock)
    data = pk.data
    for s in blk.subs:   # every sub-block is a view into the result array
        assert np.shares_memory(s.mat, data)
    before = data.copy()
    blk.subs[0].mat[0, 0] += 1.0   # an in-place change is the packed data's change
    assert blk.pack() is pk and data[np.flatnonzero(data != before)].size == 1
    blk.subs[0].mat = np.asfortranarray(blk.subs[0].mat * 2.0)   # a replaced sub-block: packed anew
    p2 = blk.pack()
    assert isinstance(p2, PackedBlock) and not np.shares_memory(p2.data, data)
    assert np.array_equal(p2.data[:blk.subs[0].mat.size], blk.subs[0].mat.reshape(-1, order="F"))


def test_model_operator_sets_built_when_read(oracle_lib):
    from oracle import oracle
    rc = synth.renorm_case("small", side=0, seed=5)
    m = oracle.get_hamiltonian(rc.lat, rc.side, rc.mshift, rc.pre, rc.basis, rc.trun)
    n = len(m.sub)
    assert n > 1 and not m.sub.built()
    pk = m.pack()
    assert pk is m._packed and not isinstance(pk, PackedModel)
    sets = list(m.sub)
    assert len(sets) == n and m.sub[-1] is sets[-1] and m.sub[1:3] == sets[1:3]
    for bs in sets:
        for k in OPS:
            for s in getattr(bs, k).subs:
                assert np.shares_memory(s.mat, pk.data)
    # the packed form agrees with a copy made from the numpy side
    fresh = PackedModel(m)
    assert fresh.c.nsub == pk.c.nsub
    for i in range(n):
        for k in OPS:
            a, b = getattr(fresh.c.sub[i], k), getattr(pk.c.sub[i], k)
            assert (a.num, a.dim) == (b.num, b.dim)
    assert m.pack() is pk
    getattr(m.sub[0], OPS[0]).subs[0].mat = np.zeros_like(getattr(m.sub[0], OPS[0]).subs[0].mat)
    assert isinstance(m.pack(), PackedModel)


def test_basis_pack_kept_while_unchanged():
    sb = synth.workload("small")
    b = sb.sys_bs
    p = b.pack()
    assert b.pack() is p and p.c.dim == b.dim
    m = b.maps[0]
    m.subs.append(m.subs[-1])   # a changed map: packed anew, with the new record
    p2 = b.pack()
    assert p2 is not p and p2.c.sub[0].num == len(m.subs)
    m.subs.pop()
    assert b.pack().c.sub[0].num == len(m.subs)
