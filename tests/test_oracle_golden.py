"""The oracle pinned against the reference's own regression output
(test/python-interface.s.ref, HF/cc-pVDZ MOLPRO dump, C2v, frozen 1s) and its
internal consistency (route 2 == route 3, batching invariance)."""
import json
import os

import numpy as np
import pytest

from binding import Oracle
from cases import SPACES, contractions_for, random_list
from gccu import H, P, occ8

GOLD = os.path.join(os.path.dirname(__file__), "golden", "hf_ccpvdz_ref.json")

# active orbitals of the fixture per C2v irrep: occupied (3,1,1,0) minus the
# frozen 1s (1,0,0,0); 19 orbitals with ORBSYM 10x1, 4x2, 4x3, 1x4
HF_NORB = [[2, 1, 1, 0], [7, 3, 3, 1], [0] * 4, [0] * 4]

H_BLOCKS = [occ8(), occ8({H: 1}, {H: 1}), occ8({H: 1}, {P: 1}), occ8({P: 1}, {H: 1}),
            occ8({P: 1}, {P: 1}), occ8({H: 2}, {H: 2}), occ8({H: 2}, {H: 1, P: 1}),
            occ8({H: 2}, {P: 2}), occ8({H: 1, P: 1}, {H: 2}), occ8({H: 1, P: 1}, {H: 1, P: 1}),
            occ8({H: 1, P: 1}, {P: 2}), occ8({P: 2}, {H: 2}), occ8({P: 2}, {H: 1, P: 1}),
            occ8({P: 2}, {P: 2})]


@pytest.fixture(scope="module")
def gold():
    with open(GOLD) as f:
        return json.load(f)


@pytest.fixture(scope="module")
def hf(built):
    return Oracle(4, HF_NORB)


def test_string_counts(gold, hf):
    # strings/set_graph2.f prints the number of strings per graph and Ms
    for g in gold["graphs"]:
        typ = g["space"] - 1
        nel = g["nel"]
        for ms, length in g["ms_len"]:
            idxms = (nel - ms) // 2 + 1
            n = sum(hf.nstr(typ, nel, idxms, gam) for gam in range(1, 5))
            assert n == length, (g, ms)


def test_list_lengths(gold, hf):
    # operators/set_op_dim2.f: len_op of the H, T2 and scalar lists
    lists = gold["lists"]
    op = hf.define_op(H_BLOCKS)
    _, n = hf.define_list(op)
    assert n == lists["H0"]["length"] == 40783
    op = hf.define_op([occ8({P: 2}, {H: 2})])
    _, n = hf.define_list(op)
    assert n == lists["ME_T2"]["length"] == lists["DIAG"]["length"] == 1134
    op = hf.define_op([occ8()])
    _, n = hf.define_list(op)
    assert n == lists["ME_LMP2"]["length"] == 1


def test_string_order_is_reverse_lexical(hf):
    # next_string order: highest orbital most significant, per orbital
    # empty < alpha < beta < pair (strings/nextstr.f)
    code = {1: 1, -1: 2, 2: 3}
    for typ, nel in ((0, 2), (1, 2), (1, 3)):
        for idxms in range(1, nel + 2):
            for gam in range(1, 5):
                orb, spn = hf.strings(typ, nel, idxms, gam)
                keys = []
                for o, s in zip(orb, spn):
                    v = [0] * 20
                    for oo, ss in zip(o, s):
                        v[oo - 1] = code[int(ss)]
                    keys.append(tuple(reversed(v)))
                assert keys == sorted(keys)


def _run_case(o, case, route, seed, **kw):
    name, op1, op2, res, ex1, ex2, cnt = case
    l1, n1 = o.define_list(o.define_op([op1]))
    l2, n2 = o.define_list(o.define_op([op2]))
    l12, n12 = o.define_list(o.define_op([res]))
    x1 = random_list(n1, seed)
    x2 = random_list(n2, seed + 1)
    x12 = random_list(n12, seed + 2)
    st = np.zeros(8)
    o.contract(route, l1, 1, x1, l2, 1, x2, l12, 1, x12, ex1, ex2, cnt, 0.75, stats=st, **kw)
    return x12, st


@pytest.mark.parametrize("space", ["c1_small", "c2v", "d2h", "c1_val"])
def test_route2_equals_route3(built, space):
    nsym, norb = SPACES[space]
    for i, case in enumerate(contractions_for(space)):
        o2 = Oracle(nsym, norb)
        o3 = Oracle(nsym, norb)
        r2, _ = _run_case(o2, case, 2, 100 + i)
        r3, st = _run_case(o3, case, 3, 100 + i)
        assert np.allclose(r2, r3, rtol=0, atol=1e-12 * max(1.0, np.abs(r2).max())), case[0]


@pytest.mark.parametrize("blocks", [(10, 100), (20, 6), (3, -1)])
def test_batching_invariance(built, blocks):
    # the reference's batch-* tests: str_block / cnt_block must not change results
    nsym, norb = SPACES["c2v"]
    for i, case in enumerate(contractions_for("c2v")):
        ra, _ = _run_case(Oracle(nsym, norb), case, 3, 7 + i)
        rb, _ = _run_case(Oracle(nsym, norb), case, 3, 7 + i, str_block=blocks[0],
                          cnt_block=blocks[1])
        assert np.allclose(ra, rb, rtol=0, atol=1e-12 * max(1.0, np.abs(ra).max())), case[0]
