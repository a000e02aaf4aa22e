"""Tile policies and the autotuner (gccu_set_tuning): every candidate policy
of both precision modes, forced, gives the oracle's results on every test
contraction of a space whose ladder blocks reach the tensor cores (its
same-spin ladder block, 276 x 15 x 276, is the thin item that one candidate
sends to the tensor cores); in autotune mode the results are the oracle's,
each new block-shape histogram is timed once, and a contraction with the
same histogram reuses the choice."""
import numpy as np
import pytest

import gccu
from binding import Oracle
from cases import contractions_for, random_list

pytestmark = pytest.mark.gpu

SPACE = (1, [[6], [24], [0], [0]])
TOL = {0: 1e-12, 1: 2e-5}
NCAND = {0: 4, 1: 6}


def _run(e, o, case, seed, mode):
    lists = []
    for occ in case[1:4]:
        le, n = e.register_list(e.define_operator([occ]))
        lo, _ = o.define_list(o.define_op([occ]))
        lists.append((le, lo, n))
    (l1, o1, n1), (l2, o2, n2), (l12, o12, n12) = lists
    x1, x2, x12 = random_list(n1, seed), random_list(n2, seed + 1), random_list(n12, seed + 2)
    e.upload(l1, x1)
    e.upload(l2, x2)
    e.upload(l12, x12)
    e.contract((l1, 1), (l2, 1), (l12, 1), case[4], case[5], case[6], fact=0.7, update=True)
    ref = x12.copy()
    o.contract(2, o1, 1, x1, o2, 1, x2, o12, 1, ref, case[4], case[5], case[6], 0.7, update=True)
    got = e.download(l12, n12)
    assert np.max(np.abs(got - ref)) <= TOL[mode] * max(1.0, np.abs(ref).max()), (case[0], mode)


@pytest.mark.parametrize("mode", [0, 1], ids=["fp64", "split_tf32"])
def test_every_candidate_matches_oracle(built, mode):
    nsym, norb = SPACE
    e = gccu.Engine(0)
    try:
        e.register_orbinfo(nsym, norb)
        e.set_precision(mode)
        for cand in range(NCAND[mode]):
            e.set_tuning(2, cand)
            o = Oracle(nsym, norb)
            for i, case in enumerate(contractions_for("c1_small")):
                _run(e, o, case, 100 * cand + 3 * i, mode)
        with pytest.raises(gccu.GccuError, match="candidate"):
            e.set_tuning(2, NCAND[mode])
    finally:
        e.close()


def test_autotune_matches_oracle_and_caches(built):
    nsym, norb = SPACE
    e = gccu.Engine(0)
    try:
        e.register_orbinfo(nsym, norb)
        e.set_precision(1)
        e.set_tuning(1)
        o = Oracle(nsym, norb)
        cases = contractions_for("c1_small")
        for i, case in enumerate(cases):
            _run(e, o, case, 7 * i, 1)
        rows = e.tuning_report()
        assert len(rows) >= 1
        assert all(0 <= r[1] < NCAND[1] for r in rows)
        # the fastest candidate, or the fixed rule when no alternative beats
        # it by more than 3%
        for r in rows:
            ms = list(r[2:2 + NCAND[1]])
            best = min(ms)
            if best >= 0.97 * ms[0]:
                assert int(r[1]) == 0 or ms[int(r[1])] == best
            else:
                assert ms[int(r[1])] == best
        # the same contractions on new lists: same histograms, no new timing
        for i, case in enumerate(cases):
            _run(e, o, case, 7 * i + 1000, 1)
        assert len(e.tuning_report()) == len(rows)
    finally:
        e.close()
