"""Partial traces (trace_op) on the host: the oracle's restatement gives the
plain trace of a one-body operator, and the engine plans every test trace."""
import numpy as np
import pytest

import gccu
from binding import Oracle
from cases import SPACES, random_list, traces_for


@pytest.mark.parametrize("space", list(SPACES))
def test_oracle_full_trace_is_the_diagonal_sum(space):
    nsym, norb = SPACES[space]
    o = Oracle(nsym, norb)
    name, op, res, cnt = traces_for(space)[0]
    assert name == "full_p"
    lo, n = o.define_list(o.define_op([op]))
    lr, nr = o.define_list(o.define_op([res]))
    assert nr == 1
    x = random_list(n, 11)
    y = np.zeros(1)
    o.trace(lo, 1, x, lr, 1, y, cnt, fac=1.0, update=False)
    # (P;P): distributions (iblk, idxmsa, gama, idxdis, offset, length, ld, did);
    # the diagonal ones (same Ms and IRREP on both sides) are square blocks
    # with C strings fastest
    ref = 0.0
    for row in o.dists(lo):
        off, ln, ld = int(row[4]), int(row[5]), int(row[6])
        if ln == ld * ld:
            blk = x[off:off + ln].reshape(ld, ld)
            ref += np.trace(blk)
    assert abs(y[0] - ref) < 1e-12


@pytest.mark.parametrize("space", list(SPACES))
def test_trace_plans(built, space):
    nsym, norb = SPACES[space]
    e = gccu.Engine(-1)
    try:
        e.register_orbinfo(nsym, norb)
        for name, op, res, cnt in traces_for(space):
            lo, _ = e.register_list(e.define_operator([op]))
            lr, _ = e.register_list(e.define_operator([res]))
            ncases, nel = e.trace_info((lo, 1), (lr, 1), cnt)
            assert ncases > 0 and nel > 0, name
    finally:
        e.close()
