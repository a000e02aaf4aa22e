"""The formula executor's item checks and intermediate arena
(gccu_formula_define, frm_sched2's command loop with [NEW] / [DEL]
intermediates, contract/frm_sched2.f:117-365), on a host-only engine: the
intermediates of overlapping [NEW] .. [DEL] windows get disjoint ranges, a
later one reuses the range of one deleted before it, and the CCSD formula's
arena is smaller than its intermediates one by one."""
import numpy as np
import pytest

import cc
import gccu
import hamiltonian as hm
from gccu import H, P, occ8


@pytest.fixture
def host_engine(built):
    e = gccu.Engine(-1)
    e.register_orbinfo(1, [[3], [5], [0], [0]])
    yield e
    e.close()


def _item(cmd, lst, **kw):
    return gccu.FormulaItem(command=cmd, list=lst, **kw)


def _add(out, src, fac=1.0, reset=1):
    return gccu.FormulaItem(command=gccu.CMD_ADD, list=out, iblk_out=1, list_in=src, iblk_in=1,
                            fac=fac, reset=reset)


def test_arena_reuses_the_ranges_of_deleted_intermediates(host_engine):
    e = host_engine
    op = e.define_operator([occ8({P: 2}, {H: 2})])
    a, n = e.register_intermediate(op)
    b, _ = e.register_intermediate(op)
    c, _ = e.register_intermediate(op)
    r, _ = e.register_list(op)
    T, NEW, DEL = gccu.CMD_TARGET, gccu.CMD_NEW, gccu.CMD_DEL
    items = [_item(NEW, a), _item(T, a), _add(a, r),
             _item(NEW, b), _item(T, b), _add(b, a), _item(DEL, a),
             _item(NEW, c), _item(T, c), _add(c, b), _item(DEL, b),
             _item(T, r), _add(r, c), _item(DEL, c)]
    fid = e.formula_define(items)
    info = e.formula_info(fid)
    size = (n * 8 + 255) // 256 * 256
    off = {x: e.intermediate_offset(x) for x in (a, b, c)}
    assert off[a] != off[b] and off[c] == off[a]
    assert info == dict(arena_bytes=2 * size, sum_bytes=3 * size, targets=4, items=len(items))


def test_formula_items_are_checked(host_engine):
    e = host_engine
    op = e.define_operator([occ8({P: 1}, {H: 1})])
    a, _ = e.register_intermediate(op)
    r, _ = e.register_list(op)
    T, NEW, DEL = gccu.CMD_TARGET, gccu.CMD_NEW, gccu.CMD_DEL
    with pytest.raises(gccu.GccuError, match="outside its"):
        e.formula_define([_item(T, r), _add(r, a)])
    with pytest.raises(gccu.GccuError, match="outside its"):
        e.formula_define([_item(NEW, a), _item(DEL, a), _item(T, r), _add(r, a)])
    with pytest.raises(gccu.GccuError, match="not an intermediate"):
        e.formula_define([_item(NEW, r)])
    with pytest.raises(gccu.GccuError, match="created once"):
        e.formula_define([_item(NEW, a), _item(DEL, a), _item(NEW, a)])
    e.formula_define([_item(NEW, a), _item(T, a), _add(a, r), _item(DEL, a)])
    with pytest.raises(gccu.GccuError, match="one formula"):
        e.formula_define([_item(NEW, a), _item(DEL, a)])


def test_ccsd_formula_arena(built):
    # the CCSD formula with its twelve intermediates created before their
    # first item and deleted after their last: the arena holds the ones
    # alive together, less than all of them (about 9% less here: tau, Y and
    # the ring W live through most of the formula)
    sp, eps, B = hm.synthetic(4, 10, 20, seed=1)
    e = gccu.Engine(-1)
    try:
        s = cc.CCSolver(e, hm.FactorizedIntegrals(sp, eps, B), method="ccsd",
                        native_formula=True)
        info = e.formula_info(s.fid)
        inter = [n for n in s.lists if n not in cc.CCSolver.PERSISTENT and
                 not n[:1] in "DSP"]
        assert len(inter) == 12
        ntarget = sum(1 for i, it in enumerate(s.formula)
                      if i == 0 or s.formula[i - 1]["res"][0] != it["res"][0])
        assert info["targets"] == ntarget
        assert info["items"] == len(s.formula) + ntarget + 2 * len(inter)
        assert info["arena_bytes"] < info["sum_bytes"], info
    finally:
        e.close()


def test_ccsdt_formula_arena(built):
    # the CCSDT formula (one intermediate per shared chain prefix, each alive
    # only while the chains of its Hamiltonian class run) through the
    # engine's item checks; the arena is a fraction of all intermediates
    sp, eps, B = hm.synthetic(3, 8, 20, seed=2)
    e = gccu.Engine(-1)
    try:
        s = cc.CCSolver(e, hm.FactorizedIntegrals(sp, eps, B), method="ccsdt",
                        native_formula=True)
        info = e.formula_info(s.fid)
        inter = [n for n in s.lists if n not in cc.CCSolver.PERSISTENT and
                 not n[:1] in "DSP"]
        assert len(inter) == sum(1 for it in s.formula if it["res"][0] in inter)
        ntarget = sum(1 for i, it in enumerate(s.formula)
                      if i == 0 or s.formula[i - 1]["res"][0] != it["res"][0])
        assert info["targets"] == ntarget
        assert info["items"] == len(s.formula) + ntarget + 2 * len(inter)
        assert info["arena_bytes"] < 0.5 * info["sum_bytes"], info
    finally:
        e.close()
