"""Singlet spin projection on the device (gccu_spin_prj_list, k_spin_prj)
against the oracle's restatement of spin_prj_list / spin_prj_blk
(contract/spin_prj_list.f, contract/spin_prj_blk.f): every test space, totally
and non-totally symmetric lists, classes with one to four creators (2 to 70
spin cases), several components per side and paired orbitals; the squared
norms per class; idempotence; the projection captured in a CUDA graph; a
closed-shell CCSD solve with its residuals projected after every evaluation
(the iterates are those of the plain solve); the reference's error cases.
Tolerance 1e-13 relative to the largest element (the device sums the
coupling products with FMA, the oracle without)."""
import numpy as np
import pytest

import cc
import gccu
import hamiltonian as hm
from binding import Oracle
from cases import SPACES, random_list
from devfill import TorchIntegrals
from gccu import H, P, V, occ8

pytestmark = pytest.mark.gpu

CLASSES = [
    occ8(),
    occ8({P: 1}, {H: 1}),
    occ8({P: 2}, {H: 2}),
    occ8({P: 3}, {H: 3}),
    occ8({P: 1, H: 1}, {P: 1, H: 1}),
    occ8({H: 2}, {H: 2}),
    occ8({P: 2}, {P: 2}),
    occ8({P: 2, H: 1}, {P: 1, H: 2}),
]
CLASSES_V = [
    occ8({P: 1, V: 1}, {H: 2}),
    occ8({P: 2}, {V: 1, H: 1}),
    occ8({P: 1, V: 1}, {H: 1, V: 1}),
    occ8({V: 2}, {V: 2}),
]
FOUR_BODY = [occ8({P: 4}, {H: 4}), occ8({P: 2, H: 2}, {P: 2, H: 2})]
TOL = 1e-13


@pytest.fixture
def engine(built):
    e = gccu.Engine(0)
    yield e
    e.close()


def _lists(engine, o, classes, gamt=1, mst=0):
    le, n = engine.register_list(engine.define_operator(classes), gamt=gamt, mst=mst)
    lo, n2 = o.define_list(o.define_op(classes), gamt=gamt, mst=mst)
    assert n == n2
    return le, lo, n


def _check(engine, o, classes, seed, gamt=1):
    le, lo, n = _lists(engine, o, classes, gamt)
    if n == 0:
        return 0
    x = random_list(n, seed)
    engine.upload(le, x)
    got_n = engine.spin_prj(le, len(classes))
    got = engine.download(le, n)
    ref = x.copy()
    ref_n = o.spin_prj(lo, ref, len(classes))
    scale = max(1.0, np.abs(ref).max())
    assert np.max(np.abs(got - ref)) <= TOL * scale
    assert np.allclose(got_n, ref_n, rtol=1e-12, atol=1e-300)
    assert np.max(np.abs(got - x)) > 1e-3 * scale  # random lists are no singlets
    engine.spin_prj(le)  # the cached plan; a projection is idempotent
    assert np.max(np.abs(engine.download(le, n) - got)) <= TOL * scale
    return n


@pytest.mark.parametrize("gamt", [1, 2])
@pytest.mark.parametrize("space", list(SPACES))
def test_spin_projection_matches_oracle(engine, space, gamt):
    nsym, norb = SPACES[space]
    if gamt > nsym:
        pytest.skip("C1 has one irrep")
    engine.register_orbinfo(nsym, norb)
    o = Oracle(nsym, norb)
    classes = CLASSES + (CLASSES_V if sum(norb[V]) > 0 else [])
    assert _check(engine, o, classes, 11 + gamt, gamt) > 0


@pytest.mark.parametrize("case", range(len(FOUR_BODY)))
def test_spin_projection_four_body_classes(engine, case):
    nsym, norb = SPACES["c1_small"]
    engine.register_orbinfo(nsym, norb)
    o = Oracle(nsym, norb)
    assert _check(engine, o, [FOUR_BODY[case]], 40 + case) > 0


def test_spin_projection_in_a_graph(engine):
    nsym, norb = SPACES["c2v"]
    engine.register_orbinfo(nsym, norb)
    o = Oracle(nsym, norb)
    le, lo, n = _lists(engine, o, CLASSES[1:4])
    x = random_list(n, 21)
    engine.upload(le, x)
    engine.spin_prj(le)  # plans
    engine.upload(le, x)
    engine.graph_begin()
    engine.spin_prj(le)
    g = engine.graph_end()
    engine.upload(le, x)
    engine.graph_launch(g)
    got = engine.download(le, n)
    ref = x.copy()
    o.spin_prj(lo, ref, 3)
    assert np.max(np.abs(got - ref)) <= TOL * max(1.0, np.abs(ref).max())


def test_ccsd_with_projected_residuals_follows_the_plain_solve(built):
    # closed-shell residuals are singlets: projecting them changes nothing
    # beyond rounding (frm_sched2 projects result lists with a spin)
    sp, eps, B = hm.synthetic(6, 30, 60, seed=6030)
    hist = {}
    for proj in (False, True):
        e = gccu.Engine(0)
        try:
            s = cc.CCSolver(e, hm.FactorizedIntegrals(sp, eps, B), method="ccsd",
                            spin_project=proj)
            s.load_hamiltonian_device(TorchIntegrals(sp, eps, B))
            s.solve(maxiter=40, conv=1e-9, use_graph=True)
            hist[proj] = s.history
        finally:
            e.close()
    assert len(hist[True]) == len(hist[False]) and hist[True][-1][2] < 1e-9
    for (_, ea, ra), (_, eb, rb) in zip(hist[False], hist[True]):
        assert abs(ea - eb) < 1e-11 and abs(ra - rb) <= 1e-11 * max(1.0, ra)


def test_spin_projection_errors(engine):
    nsym, norb = SPACES["c1_small"]
    engine.register_orbinfo(nsym, norb)
    o = Oracle(nsym, norb)
    le, _, n = _lists(engine, o, [occ8({P: 1}, {H: 2})])
    with pytest.raises(gccu.GccuError, match="particle-conserving"):
        engine.spin_prj(le)
    le, _, n = _lists(engine, o, [occ8({P: 2}, {H: 2})])
    with pytest.raises(gccu.GccuError, match="singlet"):
        engine.spin_prj(le, s2=2)
    le, _, n = _lists(engine, o, [occ8({P: 1, H: 1}, {P: 1, H: 1})], mst=2)
    with pytest.raises(gccu.GccuError, match="ms"):
        engine.spin_prj(le)
    le, _, n = _lists(engine, o, [occ8({P: 5}, {H: 5})])
    with pytest.raises(gccu.GccuError, match="at most four"):
        engine.spin_prj(le)
