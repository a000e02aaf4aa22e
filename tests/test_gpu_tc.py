"""Split-TF32 tensor-core contractions (gccu_set_precision(1)) against the
oracle's FP64 route 2: every test contraction on the test spaces plus a
larger C1 space (6 holes, 24 particles) whose ladders and rings have
hundreds of rows, columns and contraction indices, so that they take the
tensor-core path (more than 32 rows and columns, at least 256 contraction
indices), to FP32-level accuracy; switching back to FP64 restores the 1e-12
agreement.  The large space adds a contraction whose result is contiguous
along the column space (its creator string comes from the second operand),
which the tensor-core epilogue scatters column-major, and the same
contractions run under spin-flip symmetry (use_tr).  The tests also check
that the tensor-core path ran: mode 1 must differ from mode 0 at the FP32
level for some contraction of the large space."""
import numpy as np
import pytest

import gccu
from binding import Oracle
from cases import H, P, SPACES, _bc, contractions_for, occ8, random_list

pytestmark = pytest.mark.gpu

RTOL_TC = 2e-5    # split TF32 (~2^-22 per product) with FP32 accumulation over <= 4096 terms
RTOL_FP64 = 1e-12

TC_SPACES = dict(SPACES, c1_tc=(1, [[6], [24], [0], [0]]))

# result (PP;HH) with the particle pair from op2 (columns, stride 1) and the
# hole pair from op1 (rows); one particle creator and annihilator contracted
TC_EXTRA = [_bc("colmajor_result", occ8(None, {H: 2}), occ8({P: 2}), occ8({P: 1}, {P: 1}))]


@pytest.fixture
def engine(built):
    e = gccu.Engine(0)
    yield e
    e.close()


@pytest.mark.parametrize("space", list(TC_SPACES))
def test_split_tf32_contractions(engine, space):
    nsym, norb = TC_SPACES[space]
    engine.register_orbinfo(nsym, norb)
    cases = (contractions_for(space) if space in SPACES
             else contractions_for("c1_small") + TC_EXTRA)
    diffs = []
    for i, case in enumerate(cases):
        o = Oracle(nsym, norb)
        ls = []
        for occ in case[1:4]:
            le, n = engine.register_list(engine.define_operator([occ]))
            lo, _ = o.define_list(o.define_op([occ]))
            ls.append((le, lo, n))
        (l1, o1, n1), (l2, o2, n2), (l12, o12, n12) = ls
        x1, x2 = random_list(n1, 10 * i), random_list(n2, 10 * i + 1)
        engine.upload(l1, x1)
        engine.upload(l2, x2)
        ref = np.zeros(n12)
        o.contract(2, o1, 1, x1, o2, 1, x2, o12, 1, ref, case[4], case[5], case[6], 0.5,
                   update=False)
        scale = max(1.0, np.abs(ref).max())
        got = {}
        for mode, tol in ((1, RTOL_TC), (0, RTOL_FP64)):
            engine.set_precision(mode)
            engine.contract((l1, 1), (l2, 1), (l12, 1), case[4], case[5], case[6], fact=0.5,
                            update=False)
            got[mode] = engine.download(l12, n12)
            assert np.max(np.abs(got[mode] - ref)) <= tol * scale, (case[0], mode)
        engine.set_precision(0)
        diffs.append(np.max(np.abs(got[1] - got[0])) / scale)
    if space == "c1_tc":
        assert max(diffs) > 1e-10, "no contraction of the large space took the tensor-core path"


def test_split_tf32_with_spin_flip_symmetry(engine):
    # use_tr on the tensor-core path: half of the Ms cases, doubled, then the
    # spin-flip symmetrisation of the result, against the oracle's route 2
    nsym, norb = TC_SPACES["c1_tc"]
    engine.register_orbinfo(nsym, norb)
    engine.set_precision(1)
    diffs = []
    try:
        for i, case in enumerate(contractions_for("c1_small")[:5] + TC_EXTRA):
            o = Oracle(nsym, norb)
            name, op1, op2, res, ex1, ex2, cnt = case
            ls = []
            for occ in (op1, op2, res):
                le, n = engine.register_list(engine.define_operator([occ]), absym=1)
                lo, _ = o.define_list(o.define_op([occ]), absym=1)
                ls.append((le, lo, n))
            (l1, o1, n1), (l2, o2, n2), (l12, o12, n12) = ls
            x1, x2 = random_list(n1, 5 * i), random_list(n2, 5 * i + 1)
            o.sym_ab(o1, 1, x1)  # spin-symmetric inputs
            o.sym_ab(o2, 1, x2)
            engine.upload(l1, x1)
            engine.upload(l2, x2)
            ref = np.zeros(n12)
            o.contract(2, o1, 1, x1, o2, 1, x2, o12, 1, ref, ex1, ex2, cnt, 1.0, use_tr=True)
            scale = max(1.0, np.abs(ref).max())
            got = {}
            for mode in (1, 0):
                engine.set_precision(mode)
                engine.contract((l1, 1), (l2, 1), (l12, 1), ex1, ex2, cnt, fact=1.0,
                                update=False, use_tr=True)
                got[mode] = engine.download(l12, n12)
            engine.set_precision(1)
            assert np.max(np.abs(got[1] - ref)) <= RTOL_TC * scale, name
            assert np.max(np.abs(got[0] - ref)) <= RTOL_FP64 * scale, name
            diffs.append(np.max(np.abs(got[1] - got[0])) / scale)
    finally:
        engine.set_precision(0)
    assert max(diffs) > 1e-10, "no spin-flip contraction took the tensor-core path"
