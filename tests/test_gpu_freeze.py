"""Frozen lists (gccu_freeze_list): contractions planned while an operand's
list is frozen make the panels they derive from it once (split TF32 panels
of tensor-core items, gathered FP64 panels of map-addressed operands) and
reuse them.  Checked against the oracle: the results with cached panels,
again after the list is unfrozen, rewritten and frozen again (the panels are
remade), writes to a frozen list are refused, and a CUDA graph captured
while the panels were cached cannot be launched after an unfreeze."""
import numpy as np
import pytest

import gccu
from binding import Oracle
from cases import H, P, _bc, contractions_for, occ8, random_list

pytestmark = pytest.mark.gpu

SPACE = (1, [[6], [24], [0], [0]])  # ladder blocks reach the tensor cores
BIG = (1, [[6], [72], [0], [0]])
TOL = {0: 1e-12, 1: 2e-5}
# a tensor-core item whose row operand is gathered through string maps in the
# split pre-pass (three particle annihilators merged from an external and
# two contracted ones)
BIGK_MAPPED = _bc("bigk_mapped", occ8({H: 1}, {P: 1}), occ8(None, {H: 2}), occ8(None, {P: 2}))


def _case(name):
    if name == "bigk_mapped":
        return BIGK_MAPPED
    return [c for c in contractions_for("c1_small") if c[0] == name][0]


def _setup(e, o, case):
    ls = []
    for occ in case[1:4]:
        le, n = e.register_list(e.define_operator([occ]))
        lo, _ = o.define_list(o.define_op([occ]))
        ls.append((le, lo, n))
    return ls


def _ref(o, ls, x1, x2, case):
    (_, o1, _), (_, o2, _), (_, o12, n12) = ls
    ref = np.zeros(n12)
    o.contract(2, o1, 1, x1, o2, 1, x2, o12, 1, ref, case[4], case[5], case[6], 1.0,
               update=False)
    return ref


def _check(got, ref, mode):
    assert np.max(np.abs(got - ref)) <= TOL[mode] * max(1.0, np.abs(ref).max())


# (contraction, operand frozen: 0 = op1, 1 = op2, precision mode, space):
# the ladder's row operand (V) and column operand (T2) split once for the
# tensor cores; a map-addressed operand gathered and split once; the
# map-addressed T2 operand of a Fock x T2 term and of a ring packed once (FP64)
CASES = [("pp_ladder", 0, 1, SPACE), ("pp_ladder", 1, 1, SPACE),
         ("bigk_mapped", 0, 1, BIG), ("fpp_t2", 1, 0, SPACE), ("ring", 1, 0, SPACE)]


@pytest.mark.parametrize("name,frozen_op,mode,space", CASES,
                         ids=[f"{c[0]}-op{c[1] + 1}-p{c[2]}" for c in CASES])
def test_cached_operand_panels(built, name, frozen_op, mode, space):
    nsym, norb = space
    case = _case(name)
    e = gccu.Engine(0)
    try:
        e.register_orbinfo(nsym, norb)
        e.set_precision(mode)
        o = Oracle(nsym, norb)
        ls = _setup(e, o, case)
        (l1, _, n1), (l2, _, n2), (l12, _, n12) = ls
        x = [random_list(n1, 1), random_list(n2, 2)]
        e.upload(l1, x[0])
        e.upload(l2, x[1])
        lf = (l1, l2)[frozen_op]
        e.freeze(lf)
        args = ((l1, 1), (l2, 1), (l12, 1), case[4], case[5], case[6])
        ref = _ref(o, ls, x[0], x[1], case)
        for _ in range(2):  # plans (makes the cached panels), then reuses them
            e.contract(*args, update=False)
            _check(e.download(l12, n12), ref, mode)
        with pytest.raises(gccu.GccuError, match="frozen"):
            e.upload(lf, x[frozen_op])
        with pytest.raises(gccu.GccuError, match="frozen"):
            e.contract((l1, 1), (l2, 1), (lf, 1), case[4], case[5], case[6])
        # the other operand changes: the cached panels stay valid
        other = 1 - frozen_op
        x[other] = random_list((n1, n2)[other], 3)
        e.upload((l1, l2)[other], x[other])
        e.contract(*args, update=False)
        _check(e.download(l12, n12), _ref(o, ls, x[0], x[1], case), mode)
        # a graph that relies on the cached panels
        e.graph_begin()
        e.contract(*args, update=False)
        gid = e.graph_end()
        e.graph_launch(gid)
        _check(e.download(l12, n12), _ref(o, ls, x[0], x[1], case), mode)
        # unfreeze, rewrite: the panels are remade while the list is unfrozen
        e.freeze(lf, False)
        with pytest.raises(gccu.GccuError, match="unfrozen"):
            e.graph_launch(gid)
        x[frozen_op] = random_list((n1, n2)[frozen_op], 4)
        e.upload(lf, x[frozen_op])
        ref = _ref(o, ls, x[0], x[1], case)
        e.contract(*args, update=False)
        _check(e.download(l12, n12), ref, mode)
        # frozen again: remade once by the next call, then cached
        x[frozen_op] = random_list((n1, n2)[frozen_op], 5)
        e.upload(lf, x[frozen_op])
        e.freeze(lf)
        ref = _ref(o, ls, x[0], x[1], case)
        for _ in range(2):
            e.contract(*args, update=False)
            _check(e.download(l12, n12), ref, mode)
    finally:
        e.close()
