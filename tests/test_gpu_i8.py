"""FP64 emulated on the int8 tensor cores (gccu_set_precision(2) and (3)):
every operand row is cut into five (mode 2) or four (mode 3) signed 8-bit
slices under the row's scale (maximum / 127), the slice products with
s + t < S are summed exactly in int32 per s + t in TMEM and combined in
FP64.  Against the oracle's FP64 route 2 relative to the largest result
element, at 1e-9 for mode 2 (about 35 bits of each operand relative to its
row's maximum; random normal operands land near 1e-10) and 1e-7 for mode 3
(28 bits; near 1e-8): every test contraction of the test spaces and of
a larger C1 space whose ladders and rings reach the tensor cores, operands
with all-zero rows, contractions over more than 4096 indices (one int32
accumulation), spin-flip symmetry, frozen (cached) operands, a CCSD solve
whose iterates follow the FP64 ones, and the pipeline's wait time-out."""
import numpy as np
import pytest

import cc
import gccu
import hamiltonian as hm
from binding import Oracle
from cases import H, P, SPACES, _bc, contractions_for, occ8, random_list
from devfill import TorchIntegrals

pytestmark = pytest.mark.gpu

RTOL = {2: 1e-9, 3: 1e-7}
MODES = [2, 3]
SPACE_TC = (1, [[6], [24], [0], [0]])
SPACES_I8 = dict(SPACES, c1_tc=SPACE_TC)
EXTRA = [_bc("colmajor_result", occ8(None, {H: 2}), occ8({P: 2}), occ8({P: 1}, {P: 1}))]
BIG_SPACE = (1, [[6], [72], [0], [0]])
BIG_K = [
    _bc("bigk_direct", occ8({H: 2}), occ8(None, {P: 1, H: 1}), occ8(None, {P: 2})),
    _bc("bigk_mapped", occ8({H: 1}, {P: 1}), occ8(None, {H: 2}), occ8(None, {P: 2})),
]


@pytest.fixture
def engine(built):
    e = gccu.Engine(0)
    yield e
    e.close()


def _lists(engine, o, case, absym=0):
    ls = []
    for occ in case[1:4]:
        le, n = engine.register_list(engine.define_operator([occ]), absym=absym)
        lo, _ = o.define_list(o.define_op([occ]), absym=absym)
        ls.append((le, lo, n))
    return ls


def _run(engine, o, case, ls, x1, x2, mode, fact=0.5, use_tr=False):
    (l1, o1, n1), (l2, o2, n2), (l12, o12, n12) = ls
    engine.upload(l1, x1)
    engine.upload(l2, x2)
    ref = np.zeros(n12)
    o.contract(2, o1, 1, x1, o2, 1, x2, o12, 1, ref, case[4], case[5], case[6], fact,
               update=False, use_tr=use_tr)
    engine.set_precision(mode)
    try:
        engine.contract((l1, 1), (l2, 1), (l12, 1), case[4], case[5], case[6], fact=fact,
                        update=False, use_tr=use_tr)
        got = engine.download(l12, n12)
    finally:
        engine.set_precision(0)
    return got, ref


@pytest.mark.parametrize("mode", MODES)
@pytest.mark.parametrize("space", list(SPACES_I8))
def test_int8_slice_contractions(engine, space, mode):
    nsym, norb = SPACES_I8[space]
    engine.register_orbinfo(nsym, norb)
    cases = (contractions_for(space) if space in SPACES
             else contractions_for("c1_small") + EXTRA)
    worst, tc_diff = 0.0, 0.0
    for i, case in enumerate(cases):
        o = Oracle(nsym, norb)
        ls = _lists(engine, o, case)
        x1, x2 = random_list(ls[0][2], 20 * i), random_list(ls[1][2], 20 * i + 1)
        got, ref = _run(engine, o, case, ls, x1, x2, mode)
        scale = max(1.0, np.abs(ref).max())
        err = np.max(np.abs(got - ref)) / scale
        assert err <= RTOL[mode], (case[0], err)
        worst = max(worst, err)
        if space == "c1_tc":
            g1, _ = _run(engine, o, case, ls, x1, x2, 1)
            tc_diff = max(tc_diff, np.max(np.abs(g1 - ref)) / scale)
    if space == "c1_tc":
        # the int8 path ran (not FP64) and is far closer to FP64 than split TF32
        assert worst > 1e-15 and tc_diff > 30 * worst, (worst, tc_diff)


@pytest.mark.parametrize("mode", MODES)
def test_int8_slices_zero_rows(engine, mode):
    # operands whose rows are entirely zero (row scale 0) next to large rows
    nsym, norb = SPACE_TC
    engine.register_orbinfo(nsym, norb)
    case = [c for c in contractions_for("c1_small") if c[0] == "pp_ladder"][0]
    o = Oracle(nsym, norb)
    ls = _lists(engine, o, case)
    n1, n2 = ls[0][2], ls[1][2]
    x1, x2 = random_list(n1, 5), random_list(n2, 6)
    x1[: n1 // 3] = 0.0
    x2[n2 // 2:] = 0.0
    x1[-10:] *= 1e6
    got, ref = _run(engine, o, case, ls, x1, x2, mode)
    assert np.max(np.abs(got - ref)) <= RTOL[mode] * max(1.0, np.abs(ref).max())


@pytest.mark.parametrize("mode", MODES)
@pytest.mark.parametrize("case", BIG_K, ids=[c[0] for c in BIG_K])
def test_int8_slices_long_contraction(engine, case, mode):
    nsym, norb = BIG_SPACE
    engine.register_orbinfo(nsym, norb)
    o = Oracle(nsym, norb)
    ls = _lists(engine, o, case)
    x1, x2 = random_list(ls[0][2], 71), random_list(ls[1][2], 72)
    got, ref = _run(engine, o, case, ls, x1, x2, mode, fact=-0.5)
    assert np.max(np.abs(got - ref)) <= RTOL[mode] * max(1.0, np.abs(ref).max())


@pytest.mark.parametrize("mode", MODES)
def test_int8_slices_spin_flip(engine, mode):
    nsym, norb = SPACE_TC
    engine.register_orbinfo(nsym, norb)
    for i, case in enumerate(contractions_for("c1_small")[:5] + EXTRA):
        o = Oracle(nsym, norb)
        ls = _lists(engine, o, case, absym=1)
        x1, x2 = random_list(ls[0][2], 30 + i), random_list(ls[1][2], 40 + i)
        o.sym_ab(ls[0][1], 1, x1)  # spin-symmetric inputs
        o.sym_ab(ls[1][1], 1, x2)
        got, ref = _run(engine, o, case, ls, x1, x2, mode, fact=1.0, use_tr=True)
        assert np.max(np.abs(got - ref)) <= RTOL[mode] * max(1.0, np.abs(ref).max()), case[0]


@pytest.mark.parametrize("mode", MODES)
def test_int8_slices_frozen_operands(engine, mode):
    # the ladder with its row operand frozen: slices and row maxima made once
    nsym, norb = SPACE_TC
    engine.register_orbinfo(nsym, norb)
    case = [c for c in contractions_for("c1_small") if c[0] == "pp_ladder"][0]
    o = Oracle(nsym, norb)
    (l1, o1, n1), (l2, o2, n2), (l12, o12, n12) = _lists(engine, o, case)
    x1, x2 = random_list(n1, 81), random_list(n2, 82)
    engine.upload(l1, x1)
    engine.freeze(l1)
    engine.set_precision(mode)
    try:
        for seed in (83, 84):  # the column operand changes, the cached slices stay
            x2 = random_list(n2, seed)
            engine.upload(l2, x2)
            engine.contract((l1, 1), (l2, 1), (l12, 1), case[4], case[5], case[6],
                            update=False)
            ref = np.zeros(n12)
            o.contract(2, o1, 1, x1, o2, 1, x2, o12, 1, ref, case[4], case[5], case[6], 1.0,
                       update=False)
            got = engine.download(l12, n12)
            assert np.max(np.abs(got - ref)) <= RTOL[mode] * max(1.0, np.abs(ref).max())
        engine.freeze(l1, False)
        x1 = random_list(n1, 85)  # rewritten and contracted again: slices remade
        engine.upload(l1, x1)
        engine.contract((l1, 1), (l2, 1), (l12, 1), case[4], case[5], case[6], update=False)
        ref = np.zeros(n12)
        o.contract(2, o1, 1, x1, o2, 1, x2, o12, 1, ref, case[4], case[5], case[6], 1.0,
                   update=False)
        got = engine.download(l12, n12)
        assert np.max(np.abs(got - ref)) <= RTOL[mode] * max(1.0, np.abs(ref).max())
    finally:
        engine.set_precision(0)


def test_int8_slices_ccsd_solve_matches_fp64(built):
    # the whole solve with every GEMM-sized contraction on the int8 slices:
    # the iterates follow the FP64 ones (energies of every iteration to 1e-9
    # Eh) down to convergence
    sp, eps, B = hm.synthetic(6, 30, 60, seed=6030)
    hist = {}
    for mode in (0, 2):
        e = gccu.Engine(0)
        try:
            s = cc.CCSolver(e, hm.FactorizedIntegrals(sp, eps, B), method="ccsd")
            s.load_hamiltonian_device(TorchIntegrals(sp, eps, B))
            e.set_precision(mode)
            s.solve(maxiter=60, conv=1e-9, use_graph=True)
            hist[mode] = s.history
        finally:
            e.close()
    assert hist[0][-1][2] < 1e-9 and hist[2][-1][2] < 1e-9
    assert len(hist[2]) == len(hist[0])
    for (_, e0, r0), (_, e2, r2) in zip(hist[0], hist[2]):
        assert abs(e2 - e0) < 1e-9
        assert abs(r2 - r0) <= 1e-10  # residual norms, down to 1e-9


@pytest.mark.parametrize("mode", MODES)
def test_int8_pipeline_wait_timeout_is_reported(engine, mode):
    nsym, norb = SPACE_TC
    engine.register_orbinfo(nsym, norb)
    case = [c for c in contractions_for("c1_small") if c[0] == "pp_ladder"][0]
    o = Oracle(nsym, norb)
    (l1, o1, n1), (l2, o2, n2), (l12, o12, n12) = _lists(engine, o, case)
    x1, x2 = random_list(n1, 91), random_list(n2, 92)
    engine.upload(l1, x1)
    engine.upload(l2, x2)
    ref = np.zeros(n12)
    o.contract(2, o1, 1, x1, o2, 1, x2, o12, 1, ref, case[4], case[5], case[6], 1.0,
               update=False)
    args = ((l1, 1), (l2, 1), (l12, 1), case[4], case[5], case[6])
    engine.set_precision(mode)
    try:
        engine.contract(*args, update=False)  # plans; runs with the default limit
        engine.sync()
        engine.set_wait_limit(0)
        engine.contract(*args, update=False)
        with pytest.raises(gccu.GccuError, match="timed out"):
            engine.sync()
        engine.set_wait_limit(-1)
        engine.sync()
        engine.contract(*args, update=False)
        got = engine.download(l12, n12)
        assert np.max(np.abs(got - ref)) <= RTOL[mode] * max(1.0, np.abs(ref).max())
    finally:
        engine.set_precision(0)


def test_four_then_five_slices_solve_reaches_fp64(built):
    # four slices while the residual norm is above 1e-7, five after it: the
    # same converged energy as FP64
    sp, eps, B = hm.synthetic(6, 30, 60, seed=6030)
    en = {}
    for label in ("fp64", "sliced"):
        e = gccu.Engine(0)
        try:
            s = cc.CCSolver(e, hm.FactorizedIntegrals(sp, eps, B), method="ccsd")
            s.load_hamiltonian_device(TorchIntegrals(sp, eps, B))
            if label == "fp64":
                en[label] = s.solve(maxiter=60, conv=1e-9, use_graph=True)
            else:
                en[label] = s.solve_mixed(maxiter=60, conv=1e-9, schedule=[(3, 1e-7), (2, None)])
            assert s.history[-1][2] < 1e-9
        finally:
            e.close()
    assert abs(en["sliced"] - en["fp64"]) < 1e-9
