"""Operands used transposed (tra_op1 / tra_op2 / tra_op1op2 of
contract/contr_op1op2_wmaps_c.f): the oracle's restatement of the
transposed addressing equals the plain contraction of explicitly transposed
copies of the lists, and the engine plans the same block contractions for
a transposed operand as for its explicit copy."""
import numpy as np
import pytest

import gccu
from binding import Oracle
from cases import SPACES, TRANSPOSES, random_list, transpose_operands, transpose_list, \
    transpose_variants


@pytest.mark.parametrize("space", list(SPACES))
def test_oracle_transposed_equals_explicit_copy(built, space):
    nsym, norb = SPACES[space]
    nrun = 0
    for i, (case, sym) in enumerate(transpose_variants(space)):
        for tra in TRANSPOSES:
            o = Oracle(nsym, norb)
            ops = transpose_operands(o, case, sym, tra, True)
            if min(op[1] for op in ops) == 0:
                continue
            xs = [random_list(op[1], 17 * i + k) for k, op in enumerate(ops)]
            xe = [transpose_list(o, op[0], op[4], x, op[2], op[3], nsym) if t else x
                  for op, x, t in zip(ops, xs, tra)]
            (s1, _, e1, _, _), (s2, _, e2, _, _), (s12, _, e12, _, _) = ops
            ex1, ex2, cnt = case[4:7]
            for route in (2, 3):
                rs, re = xs[2].copy(), xe[2].copy()
                o.contract(route, s1, 1, xs[0], s2, 1, xs[1], s12, 1, rs, ex1, ex2, cnt, 0.75,
                           tra=tra)
                o.contract(route, e1, 1, xe[0], e2, 1, xe[1], e12, 1, re, ex1, ex2, cnt, 0.75)
                got = transpose_list(o, s12, ops[2][4], rs, e12, ops[2][3], nsym) if tra[2] \
                    else rs
                assert np.max(np.abs(got - re)) <= 1e-12 * max(1.0, np.abs(re).max()), \
                    (case[0], sym, tra, route)
            nrun += 1
    assert nrun > 0


@pytest.mark.parametrize("space", list(SPACES))
def test_engine_plans_transposed_like_explicit_copy(built, space):
    nsym, norb = SPACES[space]
    e = gccu.Engine(-1)
    try:
        e.register_orbinfo(nsym, norb)
        for case, sym in transpose_variants(space):
            for tra in TRANSPOSES:
                ops = transpose_operands(e, case, sym, tra, False)
                if min(op[1] for op in ops) == 0:
                    continue
                ex1, ex2, cnt = case[4:7]
                n_t, st_t = e.plan_info(*[(op[0], 1) for op in ops], ex1, ex2, cnt, tra=tra)
                n_e, st_e = e.plan_info(*[(op[2], 1) for op in ops], ex1, ex2, cnt)
                assert n_t == n_e and np.array_equal(st_t, st_e), (case[0], sym, tra)
    finally:
        e.close()


# classes of transposed [ADD]s: (output occupation); the input class is its
# adjoint
ADD_CLASSES = [gccu.occ8({gccu.P: 1}, {gccu.H: 1}), gccu.occ8({gccu.P: 2}, {gccu.H: 2}),
               gccu.occ8({gccu.P: 1, gccu.H: 1}, {gccu.P: 1, gccu.H: 1}),
               gccu.occ8({gccu.P: 1}, {gccu.P: 1}), gccu.occ8({gccu.P: 2}, {gccu.P: 1, gccu.H: 1})]


def add_transp_variants(space):
    nsym = SPACES[space][0]
    for occ in ADD_CLASSES:
        yield occ, (1, 0)
        if nsym > 1:
            yield occ, (2, 0)
        yield occ, (1, 2)


def _pure_excitation(occ):
    # no hpvx type among both the creators and the annihilators
    return not any(occ[t] > 0 and occ[4 + t] > 0 for t in range(4))


@pytest.mark.parametrize("space", list(SPACES))
def test_oracle_add_transp_equals_explicit_copy(built, space):
    # add_opblk_transp (contract/add_opblk_transp.f) with tra_in:
    # out(IC,IA) += fac * in(IA,IC), against the explicitly transposed copy of
    # the input list.  With tra_out the output is addressed in set_op_ldim_c's
    # A-C sequence, which for pure (de)excitation classes is the C-A one
    # (contract/set_op_ldim_c.f:24-25): the same result there
    from cases import cnt_dag
    nsym, norb = SPACES[space]
    nrun = 0
    for i, (occ, (g, m)) in enumerate(add_transp_variants(space)):
        for tra_in, tra_out in ((1, 0), (0, 1)):
            if tra_out and not _pure_excitation(occ):
                continue
            o = Oracle(nsym, norb)
            lo, no = o.define_list(o.define_op([occ]), g, m)
            li, ni = o.define_list(o.define_op([cnt_dag(occ)]), g, -m)
            if no == 0:
                continue
            xin, xout = random_list(ni, 3 * i), random_list(no, 3 * i + 1)
            ref = xout + 0.6 * transpose_list(o, li, cnt_dag(occ), xin, lo, no, nsym)
            got = xout.copy()
            xn = o.add_transp(0.6, li, 1, xin, lo, 1, got, tra_in, tra_out)
            assert np.max(np.abs(got - ref)) <= 1e-14 * max(1.0, np.abs(ref).max())
            assert xn == pytest.approx(float(ref @ ref), rel=1e-12)
            nrun += 1
    assert nrun > 0
