"""Product host logic (host-only engine, no device) against the oracle:
lexical string addresses, ME-list layouts and the block-contraction plan."""
import numpy as np
import pytest

import gccu
from binding import Oracle
from cases import SPACES, contractions_for, random_list
from gccu import H, occ8
from test_oracle_golden import H_BLOCKS, _run_case


@pytest.fixture
def host_engine(built):
    e = gccu.Engine(-1)
    yield e
    e.close()


@pytest.mark.parametrize("space", list(SPACES))
def test_addresses_match_enumeration(host_engine, space):
    nsym, norb = SPACES[space]
    o = Oracle(nsym, norb)
    host_engine.register_orbinfo(nsym, norb)
    for typ in range(3):
        for nel in (1, 2, 3):
            for idxms in range(1, nel + 2):
                for gam in range(1, nsym + 1):
                    n = o.nstr(typ, nel, idxms, gam)
                    assert host_engine.nstr(typ, nel, idxms, gam) == n
                    orb, spn = o.strings(typ, nel, idxms, gam)
                    for i in range(n):
                        assert host_engine.string_index(typ, orb[i], spn[i]) == i


@pytest.mark.parametrize("space", list(SPACES))
def test_layout_matches_oracle(host_engine, space):
    nsym, norb = SPACES[space]
    o = Oracle(nsym, norb)
    host_engine.register_orbinfo(nsym, norb)
    ops = [H_BLOCKS] + [[c[k]] for c in contractions_for(space) for k in (1, 2, 3)]
    for occs in ops:
        for gamt in (1, nsym):
            lo, no = o.define_list(o.define_op(occs), gamt=gamt)
            le, ne = host_engine.register_list(host_engine.define_operator(occs), gamt=gamt)
            assert no == ne
            assert np.array_equal(o.dists(lo), host_engine.dists(le))


@pytest.mark.parametrize("space", list(SPACES))
def test_plan_matches_oracle_enumeration(host_engine, space):
    # the planner's block contractions, counted in the reference's dgemm
    # accounting, equal the blocks the oracle enumerates (random, unscreened data)
    nsym, norb = SPACES[space]
    host_engine.register_orbinfo(nsym, norb)
    for i, case in enumerate(contractions_for(space)):
        name, op1, op2, res, ex1, ex2, cnt = case
        l1, _ = host_engine.register_list(host_engine.define_operator([op1]))
        l2, _ = host_engine.register_list(host_engine.define_operator([op2]))
        l12, _ = host_engine.register_list(host_engine.define_operator([res]))
        nitems, st = host_engine.plan_info((l1, 1), (l2, 1), (l12, 1), ex1, ex2, cnt)
        _, sto = _run_case(Oracle(nsym, norb), case, 3, 11 + i)
        assert np.array_equal(st, sto), (name, st, sto)


@pytest.mark.parametrize("space", list(SPACES))
def test_plan_items_agree_with_plan_info(host_engine, space):
    # gccu_plan_items lists the same block contractions gccu_plan_info counts;
    # their 2*M*N*K sums to the reference's dgemm flop accounting, and the
    # map-component counts are those of the operands' string merges
    nsym, norb = SPACES[space]
    host_engine.register_orbinfo(nsym, norb)
    for case in contractions_for(space):
        name, op1, op2, res, ex1, ex2, cnt = case
        ls = [host_engine.register_list(host_engine.define_operator([o]))[0]
              for o in (op1, op2, res)]
        args = [(l, 1) for l in ls] + [ex1, ex2, cnt]
        nitems, st = host_engine.plan_info(*args)
        rows = host_engine.plan_items(*args)
        assert len(rows) == nitems, name
        assert (rows[:, :3] > 0).all(), name
        assert 2.0 * float(np.sum(rows[:, 0] * rows[:, 1] * rows[:, 2])) == st[7], name
        assert ((rows[:, 3:6] >= 0) & (rows[:, 3:6] <= 8)).all(), name


def test_contraction_descriptors_are_checked(host_engine):
    # a [CONTR] whose occupations, class indices or symmetries do not fit its
    # lists is refused with the reason, as the reference quits on them
    # (contract/contr_op1op2_wmaps_c.f)
    nsym, norb = SPACES["c2v"]
    host_engine.register_orbinfo(nsym, norb)
    name, op1, op2, res, ex1, ex2, cnt = [c for c in contractions_for("c2v")
                                          if c[0] == "ring"][0]
    l1, l2, l12 = [host_engine.register_list(host_engine.define_operator([o]))[0]
                   for o in (op1, op2, res)]
    ok = [(l1, 1), (l2, 1), (l12, 1)]
    assert host_engine.plan_info(*ok, ex1, ex2, cnt)[0] > 0
    with pytest.raises(gccu.GccuError, match="op1 occupation"):
        host_engine.plan_info(*ok, ex1 + np.eye(8, dtype=np.int64)[1], ex2, cnt)
    with pytest.raises(gccu.GccuError, match="bad op1 block"):
        host_engine.plan_info((l1, 2), (l2, 1), (l12, 1), ex1, ex2, cnt)
    with pytest.raises(gccu.GccuError, match="bad result block"):
        host_engine.plan_info((l1, 1), (l2, 1), (l12, 0), ex1, ex2, cnt)
    l12b, _ = host_engine.register_list(host_engine.define_operator([res]), gamt=2)
    with pytest.raises(gccu.GccuError, match="inconsistent symmetries"):
        host_engine.plan_info((l1, 1), (l2, 1), (l12b, 1), ex1, ex2, cnt)


def test_contraction_of_an_empty_class_plans_nothing(host_engine):
    # seven holes do not fit the six hole spin orbitals of c1_small: the
    # classes of op1 and of the result are empty, the contraction plans no
    # block contraction
    nsym, norb = SPACES["c1_small"]
    host_engine.register_orbinfo(nsym, norb)
    ex1, ex2, cnt = occ8({H: 6}, {H: 7}), occ8({H: 1}), occ8({H: 1})
    op1 = np.asarray(ex1) + np.asarray(cnt)
    op2 = np.asarray(occ8({H: 1}, {H: 1}))
    res = np.asarray(ex1) + np.asarray(ex2)
    (l1, n1), (l2, n2), (l12, n12) = [host_engine.register_list(host_engine.define_operator([o]))
                                      for o in (op1, op2, res)]
    assert n1 == 0 and n12 == 0 and n2 > 0
    n, st = host_engine.plan_info((l1, 1), (l2, 1), (l12, 1), ex1, ex2, cnt)
    assert n == 0 and not np.any(st)
