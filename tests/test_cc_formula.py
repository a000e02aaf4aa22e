"""The CC drivers (formula items + solver) on the CPU oracle against the
reference's golden MP2 run and a dense spin-orbital CCSD."""
import json
import os

import numpy as np
import pytest

import cc
import dense_cc
import hamiltonian as hm
from engine import OracleEngine

GOLD = os.path.join(os.path.dirname(__file__), "golden")


@pytest.fixture(scope="module")
def hf_ints():
    d = hm.read_fcidump(os.path.join(GOLD, "hf_ccpvdz_fcidump.npz"))
    sp = hm.OrbitalSpace(d["orbsym"], [3, 1, 1, 0], [1, 0, 0, 0])
    f = hm.fock(d["h"], d["eri"], sp.occ_all)
    return hm.DenseIntegrals(sp, f, d["eri"])


@pytest.fixture(scope="module")
def gold():
    return json.load(open(os.path.join(GOLD, "hf_ccpvdz_ref.json")))


def test_dense_mp2_matches_reference(hf_ints, gold):
    sp, f, eri = hf_ints.space, hf_ints.f, hf_ints.eri
    o, v = sp.hole, sp.part
    eo, ev = np.diag(f)[o], np.diag(f)[v]
    iajb = eri[np.ix_(o, v, o, v)]
    D = eo[:, None, None, None] - ev[None, :, None, None] + eo[None, None, :, None] - \
        ev[None, None, None, :]
    e = np.sum(iajb * (2 * iajb - iajb.transpose(0, 3, 2, 1)) / D)
    assert abs(e + gold["lmp2_norm"]) < 1e-13


@pytest.mark.parametrize("route", [2, 3])
def test_mp2_through_contractions_matches_reference(hf_ints, gold, route):
    # the reference prints ">>> 1 0.000000000000 1.100" and then
    # ">>> 2 -0.196151291382 0.6566E-14" (test/python-interface.s.ref:583,627)
    s = cc.CCSolver(OracleEngine(route=route), hf_ints, method="mp2")
    s.load_hamiltonian()
    e = s.solve(maxiter=5, conv=1e-10)
    (i1, e1, r1), (i2, e2, r2) = s.history[:2]
    assert e1 == 0.0 and round(r1, 3) == 1.100
    assert abs(e2 - gold["final_energy_12digits"]) < 1e-12
    assert abs(e + gold["lmp2_norm"]) < 1e-13
    assert r2 < 1e-13


def test_ccsd_formula_matches_dense(hf_ints):
    F, W, no = dense_cc.spin_orbital(hf_ints.space, hf_ints.f, hf_ints.eri_elems)
    _, hd = dense_cc.ccsd(F, W, no, maxiter=5)
    s = cc.CCSolver(OracleEngine(route=3), hf_ints, method="ccsd")
    s.load_hamiltonian()
    s.solve(maxiter=5, conv=1e-12, diis=False)
    for (i, ed, rd), (j, eo, ro) in zip(hd, s.history):
        assert abs(ed - eo) < 1e-12 and abs(rd - ro) < 1e-11 * max(1, rd), (i, ed, eo, rd, ro)


def test_ccsd_synthetic_c1(built):
    # a seeded synthetic Hamiltonian of the benchmark family, o=3 v=6
    sp, eps, B = hm.synthetic(3, 6, 20, seed=3)
    ints = hm.FactorizedIntegrals(sp, eps, B)
    dense = hm.DenseIntegrals(sp, np.diag(eps), ints.dense_eri())
    F, W, no = dense_cc.spin_orbital(sp, dense.f, dense.eri_elems)
    ed, hd = dense_cc.ccsd(F, W, no, maxiter=30, conv=1e-9)
    s = cc.CCSolver(OracleEngine(route=3), ints, method="ccsd")
    s.load_hamiltonian()
    eo = s.solve(maxiter=30, conv=1e-9)
    assert abs(ed - eo) < 1e-10


def test_ccsd_spin_flip_symmetry_same_iterates(hf_ints):
    # use_tr (calculate.routes.use_tr, the reference's default): every
    # contraction computes half of its Ms cases into spin-symmetric lists,
    # doubled, then symmetrised (sym_ab_blk); the iterates equal those of the
    # plain evaluation
    hist = []
    for use_tr in (False, True):
        s = cc.CCSolver(OracleEngine(route=3), hf_ints, method="ccsd", use_tr=use_tr)
        s.load_hamiltonian()
        s.solve(maxiter=6, conv=1e-14)
        hist.append(s.history)
    for (i, ea, ra), (_, eb, rb) in zip(*hist):
        assert abs(ea - eb) < 1e-12 and abs(ra - rb) < 1e-11 * max(1.0, ra), (i, ea, eb)


def test_ccsd_synthetic_d2h(built):
    # the benchmark family in D2h (irreps round-robin over orbitals and
    # auxiliary functions, integrals not totally symmetric zeroed): the
    # symmetry-blocked lists give the dense CCSD energy
    sp, eps, B = hm.synthetic(4, 8, 24, seed=8, nsym=8)
    assert sp.nsym == 8
    ints = hm.FactorizedIntegrals(sp, eps, B)
    dense = hm.DenseIntegrals(sp, np.diag(eps), ints.dense_eri())
    F, W, no = dense_cc.spin_orbital(sp, dense.f, dense.eri_elems)
    ed, hd = dense_cc.ccsd(F, W, no, maxiter=40, conv=1e-9)
    s = cc.CCSolver(OracleEngine(route=3), ints, method="ccsd")
    s.load_hamiltonian()
    eo = s.solve(maxiter=40, conv=1e-9)
    assert abs(ed - eo) < 1e-10


def test_ccsd_residuals_of_a_closed_shell_are_singlets(hf_ints):
    # the residual lists of a spin-free Hamiltonian and singlet amplitudes are
    # singlet operators: projecting them (spin_prj_list, which frm_sched2
    # applies to result lists with a spin at the end of each target) leaves
    # the iterates of the reference's HF/cc-pVDZ case unchanged; residuals of
    # amplitudes with a triplet part do change
    hist = []
    for proj in (False, True):
        s = cc.CCSolver(OracleEngine(route=3), hf_ints, method="ccsd", spin_project=proj)
        s.load_hamiltonian()
        s.solve(maxiter=6, conv=1e-14)
        hist.append(s.history)
    for (i, ea, ra), (_, eb, rb) in zip(*hist):
        assert abs(ea - eb) < 1e-12 and abs(ra - rb) < 1e-11 * max(1.0, ra), (i, ea, eb)
    for a in ("R1", "R2"):
        r = s.e.data[s.lid(a)].copy()
        s.e.spin_prj(s.lid(a))
        assert np.abs(s.e.data[s.lid(a)] - r).max() <= 1e-13 * np.abs(r).max(), a
    t2 = s.lid("T2")
    s.e.data[t2] += 1e-3 * np.random.default_rng(5).standard_normal(s.e.data[t2].shape)
    s.evaluate()
    r2 = s.e.data[s.lid("R2")].copy()
    s.project_residuals()
    moved = np.abs(s.e.data[s.lid("R2")] - r2).max()
    assert moved > 1e-6 * np.abs(r2).max()


def test_fcidump_filled_through_the_device_path_equals_host_fill(hf_ints, gold):
    # the FCIDUMP's records scattered into h and (pq|rs) by torch, the Fock
    # matrix and the lists formed from them (the device path, here with torch
    # on the CPU): the same lists as the host fill and the reference's MP2
    # energy
    from devfill import TorchDenseIntegrals
    path = os.path.join(GOLD, "hf_ccpvdz_fcidump.npz")
    tints = TorchDenseIntegrals.from_fcidump(path, [3, 1, 1, 0], [1, 0, 0, 0], device="cpu")
    host = cc.CCSolver(OracleEngine(route=3), hf_ints, method="mp2")
    host.load_hamiltonian()
    dev = cc.CCSolver(OracleEngine(route=3), tints, method="mp2")
    dev.load_hamiltonian_device(tints)
    for name in ("F", "V", "DT2"):
        a, b = host.e.data[host.lid(name)], dev.e.data[dev.lid(name)]
        assert np.max(np.abs(a - b)) <= 1e-13 * max(1.0, np.abs(a).max()), name
    e = dev.solve(maxiter=5, conv=1e-10)
    assert abs(e + gold["lmp2_norm"]) < 1e-13
