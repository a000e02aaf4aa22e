"""GPU parity of partial traces (self-contractions, trace_op): gccu_trace
against the oracle's restatement of trace_op / trace_op_blk, to 1e-12
relative, with and without update."""
import numpy as np
import pytest

import gccu
from binding import Oracle
from cases import SPACES, random_list, traces_for

pytestmark = pytest.mark.gpu

RTOL = 1e-12


@pytest.fixture
def engine(built):
    e = gccu.Engine(0)
    yield e
    e.close()


@pytest.mark.parametrize("space", list(SPACES))
def test_trace_matches_oracle(engine, space):
    nsym, norb = SPACES[space]
    engine.register_orbinfo(nsym, norb)
    for i, (name, op, res, cnt) in enumerate(traces_for(space)):
        o = Oracle(nsym, norb)
        le1, n1 = engine.register_list(engine.define_operator([op]))
        le2, n2 = engine.register_list(engine.define_operator([res]))
        lo1, no1 = o.define_list(o.define_op([op]))
        lo2, no2 = o.define_list(o.define_op([res]))
        assert (n1, n2) == (no1, no2)
        for update in (True, False):
            x = random_list(n1, 50 * i + 1)
            y = random_list(n2, 50 * i + 2)
            engine.upload(le1, x)
            engine.upload(le2, y)
            ref = y.copy()
            o.trace(lo1, 1, x, lo2, 1, ref, cnt, fac=-1.5, update=update)
            nrm = engine.trace((le1, 1), (le2, 1), cnt, fact=-1.5, update=update, xret=1)
            got = engine.download(le2, n2)
            scale = max(1.0, np.abs(ref).max())
            assert np.max(np.abs(got - ref)) <= RTOL * scale, (name, update)
            assert abs(nrm - float(ref @ ref)) <= 1e-10 * max(1.0, float(ref @ ref)), name
