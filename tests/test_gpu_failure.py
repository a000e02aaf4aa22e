"""Failure detection of the tensor-core pipeline without a GPU fault: with
the wait limit set to zero every mbarrier wait of the split-TF32 GEMM gives
up at once; the kernel waits for the work it has issued, frees its TMEM,
sets the engine's error flag and returns.  The next synchronising call
reports the time-out, and with the default limit restored the same
contraction runs clean and matches the oracle."""
import numpy as np
import pytest

import gccu
from binding import Oracle
from cases import contractions_for, random_list

pytestmark = pytest.mark.gpu

RTOL_TC = 2e-5
SPACE = (1, [[6], [24], [0], [0]])  # ladder blocks large enough for the tensor cores


def test_pipeline_wait_timeout_is_reported(built):
    nsym, norb = SPACE
    case = [c for c in contractions_for("c1_small") if c[0] == "pp_ladder"][0]
    e = gccu.Engine(0)
    try:
        e.register_orbinfo(nsym, norb)
        o = Oracle(nsym, norb)
        ls = []
        for occ in case[1:4]:
            le, n = e.register_list(e.define_operator([occ]))
            lo, _ = o.define_list(o.define_op([occ]))
            ls.append((le, lo, n))
        (l1, o1, n1), (l2, o2, n2), (l12, o12, n12) = ls
        x1, x2 = random_list(n1, 41), random_list(n2, 42)
        e.upload(l1, x1)
        e.upload(l2, x2)
        ref = np.zeros(n12)
        o.contract(2, o1, 1, x1, o2, 1, x2, o12, 1, ref, case[4], case[5], case[6], 1.0,
                   update=False)
        scale = max(1.0, np.abs(ref).max())
        args = ((l1, 1), (l2, 1), (l12, 1), case[4], case[5], case[6])
        e.set_precision(1)
        e.contract(*args, update=False)  # plans; runs with the default limit
        e.sync()
        plan = e.plan_items(*args)
        assert (plan[:, 2] >= 256).any() and (plan[:, 1] > 32).any()  # tensor-core items
        e.set_wait_limit(0)
        e.contract(*args, update=False)
        with pytest.raises(gccu.GccuError, match="timed out"):
            e.sync()
        e.set_wait_limit(-1)
        e.sync()  # the flag was cleared when it was reported
        e.contract(*args, update=False)
        got = e.download(l12, n12)
        assert np.max(np.abs(got - ref)) <= RTOL_TC * scale
    finally:
        e.close()
