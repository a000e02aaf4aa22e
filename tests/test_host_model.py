"""Product host logic (host-only engine, no device) against the oracle:
lexical string addresses, ME-list layouts and the block-contraction plan."""
import numpy as np
import pytest

import gccu
from binding import Oracle
from cases import SPACES, contractions_for, random_list
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


@pytest.mark.parametrize("space", ["c1_small", "c2v", "d2h"])
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


@pytest.mark.parametrize("space", ["c1_small", "c2v", "d2h"])
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
