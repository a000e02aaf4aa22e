"""GPU parity of [REORDER] on joined (multi-vertex) operators: gccu_reorder
against the oracle's restatement of reo_op_wmaps_c / reo_blk_wmaps_c, to
1e-12 relative, with and without update and with both reorder signs."""
import numpy as np
import pytest

import gccu
from binding import Oracle
from cases import SPACES, random_list, reorders_for

pytestmark = pytest.mark.gpu

RTOL = 1e-12


@pytest.fixture
def engine(built):
    e = gccu.Engine(0)
    yield e
    e.close()


@pytest.mark.parametrize("space", list(SPACES))
def test_reorder_matches_oracle(engine, space):
    nsym, norb = SPACES[space]
    engine.register_orbinfo(nsym, norb)
    for i, (name, nj, ori, reo, shifts) in enumerate(reorders_for(space)):
        o = Oracle(nsym, norb)
        lists = []
        for vertices in (ori, reo):
            occ = np.stack(vertices)
            le, n = engine.register_list(engine.define_operator_joined(occ, nj))
            lo, no = o.define_list(o.define_op_joined(occ, nj))
            assert n == no
            lists.append((le, lo, n))
        (le1, lo1, n1), (le2, lo2, n2) = lists
        for update, sign in ((True, 1), (False, -1)):
            x = random_list(n1, 100 * i + 3)
            y = random_list(n2, 100 * i + 4)
            engine.upload(le1, x)
            engine.upload(le2, y)
            ref = y.copy()
            o.reorder(lo1, 1, x, lo2, 1, ref, shifts, fac=0.75, sign_reo=sign, update=update)
            nrm = engine.reorder((le1, 1), (le2, 1), shifts, fac=0.75, sign_reo=sign,
                                 update=update, xret=1)
            got = engine.download(le2, n2)
            scale = max(1.0, np.abs(ref).max())
            assert np.max(np.abs(got - ref)) <= RTOL * scale, (name, update)
            assert abs(nrm - float(ref @ ref)) <= 1e-10 * max(1.0, float(ref @ ref)), name


def test_joined_operands_rejected_by_contract(engine):
    nsym, norb = SPACES["c2v"]
    engine.register_orbinfo(nsym, norb)
    name, nj, ori, reo, shifts = reorders_for("c2v")[1]
    lj, _ = engine.register_list(engine.define_operator_joined(np.stack(ori), nj))
    l1, _ = engine.register_list(engine.define_operator([gccu.occ8({gccu.P: 1}, {gccu.H: 1})]))
    with pytest.raises(gccu.GccuError, match="joined"):
        engine.contract((lj, 1), (l1, 1), (l1, 1), gccu.occ8(), gccu.occ8(),
                        gccu.occ8({gccu.P: 1}, {gccu.H: 1}))
