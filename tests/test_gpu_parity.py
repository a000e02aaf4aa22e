"""GPU parity: the device string maps are bit-exact with the oracle's
set_strmap_kernel restatement, and every block contraction matches the
oracle's route-2 scalar kernel to 1e-12 relative (FP64 path)."""
import numpy as np
import pytest

import gccu
from binding import Oracle, add_opblk, diavc
from cases import SPACES, contractions_for, random_list

pytestmark = pytest.mark.gpu

RTOL = 1e-12  # FP64 path: per-block agreement with the reference kernel


@pytest.fixture
def engine(built):
    e = gccu.Engine(0)
    yield e
    e.close()


@pytest.mark.parametrize("space", list(SPACES))
def test_strmap_bit_exact(engine, space):
    nsym, norb = SPACES[space]
    o = Oracle(nsym, norb)
    engine.register_orbinfo(nsym, norb)
    nblocks = 0
    for typ in range(3):
        for n1, n2 in ((1, 1), (1, 2), (2, 1), (2, 2), (1, 3)):
            for ix1 in range(1, n1 + 2):
                for ix2 in range(1, n2 + 2):
                    for g1 in range(1, nsym + 1):
                        for g2 in range(1, nsym + 1):
                            a = o.strmap(typ, n1, n2, ix1, ix2, g1, g2)
                            b = engine.strmap(typ, n1, n2, ix1, ix2, g1, g2)
                            assert np.array_equal(a, b), (typ, n1, n2, ix1, ix2, g1, g2)
                            nblocks += a.size > 0
    assert nblocks > 0


def _lists(e, o, case):
    name, op1, op2, res, ex1, ex2, cnt = case
    out = []
    for occ in (op1, op2, res):
        le, n = e.register_list(e.define_operator([occ]))
        lo, no = o.define_list(o.define_op([occ]))
        assert n == no
        out.append((le, lo, n))
    return out


@pytest.mark.parametrize("space", list(SPACES))
@pytest.mark.parametrize("update", [True, False])
def test_contractions_match_oracle(engine, space, update):
    nsym, norb = SPACES[space]
    engine.register_orbinfo(nsym, norb)
    for i, case in enumerate(contractions_for(space)):
        o = Oracle(nsym, norb)
        (l1, o1, n1), (l2, o2, n2), (l12, o12, n12) = _lists(engine, o, case)
        x1, x2, x12 = (random_list(n1, 10 * i), random_list(n2, 10 * i + 1),
                       random_list(n12, 10 * i + 2))
        engine.upload(l1, x1)
        engine.upload(l2, x2)
        engine.upload(l12, x12)
        ref = x12.copy()
        o.contract(2, o1, 1, x1, o2, 1, x2, o12, 1, ref, case[4], case[5], case[6], -1.25,
                   update=update)
        nrm = engine.contract((l1, 1), (l2, 1), (l12, 1), case[4], case[5], case[6], fact=-1.25,
                              update=update, xret=1)
        got = engine.download(l12, n12)
        scale = max(1.0, np.abs(ref).max())
        assert np.max(np.abs(got - ref)) <= RTOL * scale, case[0]
        assert abs(nrm - float(ref @ ref)) <= 1e-10 * max(1.0, float(ref @ ref))


def test_contraction_reuse_and_graph(engine):
    # plans are cached: the same [CONTR] twice, then replayed from a CUDA graph
    nsym, norb = SPACES["c2v"]
    engine.register_orbinfo(nsym, norb)
    case = contractions_for("c2v")[4]
    o = Oracle(nsym, norb)
    (l1, o1, n1), (l2, o2, n2), (l12, o12, n12) = _lists(engine, o, case)
    x1, x2 = random_list(n1, 5), random_list(n2, 6)
    engine.upload(l1, x1)
    engine.upload(l2, x2)
    engine.zero(l12)
    ref = np.zeros(n12)
    args = ((l1, 1), (l2, 1), (l12, 1), case[4], case[5], case[6])
    engine.contract(*args, fact=0.5)
    engine.graph_begin()
    engine.contract(*args, fact=0.5)
    engine.contract(*args, fact=0.5)
    g = engine.graph_end()
    engine.graph_launch(g)
    engine.sync()
    for _ in range(3):
        o.contract(2, o1, 1, x1, o2, 1, x2, o12, 1, ref, case[4], case[5], case[6], 0.5)
    got = engine.download(l12, n12)
    assert np.max(np.abs(got - ref)) <= RTOL * max(1.0, np.abs(ref).max())


def test_use_tr_matches_oracle(engine):
    # spin-flip symmetry (use_tr): half the Ms cases, doubled, then sym_ab_blk
    nsym, norb = SPACES["c2v"]
    engine.register_orbinfo(nsym, norb)
    for i, case in enumerate(contractions_for("c2v")[:5]):
        o = Oracle(nsym, norb)
        name, op1, op2, res, ex1, ex2, cnt = case
        lists = []
        for occ in (op1, op2, res):
            le, n = engine.register_list(engine.define_operator([occ]), absym=1)
            lo, _ = o.define_list(o.define_op([occ]), absym=1)
            lists.append((le, lo, n))
        (l1, o1, n1), (l2, o2, n2), (l12, o12, n12) = lists
        # spin-symmetric inputs: symmetrise random data with the oracle
        x1, x2 = random_list(n1, 3 * i), random_list(n2, 3 * i + 1)
        o.sym_ab(o1, 1, x1)
        o.sym_ab(o2, 1, x2)
        engine.upload(l1, x1)
        engine.upload(l2, x2)
        engine.zero(l12)
        ref = np.zeros(n12)
        o.contract(2, o1, 1, x1, o2, 1, x2, o12, 1, ref, ex1, ex2, cnt, 1.0, use_tr=True)
        full = np.zeros(n12)
        o.contract(2, o1, 1, x1, o2, 1, x2, o12, 1, full, ex1, ex2, cnt, 1.0, use_tr=False)
        assert np.allclose(ref, full, atol=1e-12 * max(1, np.abs(full).max())), name
        engine.contract((l1, 1), (l2, 1), (l12, 1), ex1, ex2, cnt, fact=1.0, use_tr=True)
        got = engine.download(l12, n12)
        assert np.max(np.abs(got - ref)) <= RTOL * max(1.0, np.abs(ref).max()), name


def test_vector_kernels(engine):
    nsym, norb = SPACES["c2v"]
    engine.register_orbinfo(nsym, norb)
    occ = contractions_for("c2v")[0][3]
    la, n = engine.register_list(engine.define_operator([occ]))
    lb, _ = engine.register_list(engine.define_operator([occ]))
    lc, _ = engine.register_list(engine.define_operator([occ]))
    a, b = random_list(n, 1), random_list(n, 2)
    d = np.abs(random_list(n, 3)) + 0.1
    d[0] = 1e-12  # clamped denominator
    engine.upload(la, a)
    engine.upload(lb, b)
    engine.upload(lc, d)
    ref = b.copy()
    xn = add_opblk(ref, a, 0.3)
    assert abs(engine.add_block(0.3, la, 1, lb, 1, typ=1) - xn) <= 1e-12 * xn
    assert np.allclose(engine.download(lb, n), ref, rtol=0, atol=1e-14)
    assert abs(engine.dot(la, lb) - float(a @ ref)) <= 1e-12 * abs(float(a @ ref)) + 1e-12
    engine.precondition(lb, la, lc, fac=-1.0, shift=0.0)
    assert np.array_equal(engine.download(lb, n), diavc(a, d, -1.0))
    engine.scale(la, 2.0)
    assert np.array_equal(engine.download(la, n), 2.0 * a)


def test_sym_ab_matches_oracle(engine):
    nsym, norb = SPACES["d2h"]
    engine.register_orbinfo(nsym, norb)
    o = Oracle(nsym, norb)
    for i, case in enumerate(contractions_for("d2h")):
        occ = case[3]
        le, n = engine.register_list(engine.define_operator([occ]), absym=1)
        lo, _ = o.define_list(o.define_op([occ]), absym=1)
        x = random_list(n, i)
        engine.upload(le, x)
        o.sym_ab(lo, 1, x, 0.5, 1.0)
        engine.sym_ab(le, 1, 0.5, 1.0)
        assert np.allclose(engine.download(le, n), x, rtol=0, atol=1e-14), case[0]
