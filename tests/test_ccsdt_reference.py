"""The reference's CCSDT regression run (test/CC-energy-I.inp: CH2/DZ from
DALTON's interface files, C2v, CC maxexc=3, frozen (1,0,0,0), deleted
(2,1,0,0), DIIS maxsub 8, conv 1e-10) reproduced through the CCSDT formula
(cc.excitation_formula) and the DIIS solver on the CPU oracle: every
iteration's energy and residual norm as the reference printed them
(test/CC-energy-I.e.ref), the iteration count and the final energy; and the
CCSD ground state of test/CC-excite-I.e.ref on the same integrals through
the CCSD formula.  Fixtures from tests/golden/make_ch2_dalton.py."""
import json
import os

import numpy as np
import pytest

import cc
import hamiltonian as hm
from engine import OracleEngine

GOLD = os.path.join(os.path.dirname(__file__), "golden")


def ch2_dz_integrals():
    """the CH2/DZ space, MO Fock matrix and (pq|rs) of the fixture"""
    d = np.load(os.path.join(GOLD, "ch2_dz_dalton.npz"))
    ref = json.load(open(os.path.join(GOLD, "ch2_dz_ccsdt_ref.json")))
    orbsym = d["orbsym"]
    n = len(orbsym)
    # symmetry-blocked packed upper triangles, column by column
    f = np.zeros((n, n))
    k = off = 0
    for g in range(1, int(orbsym.max()) + 1):
        m = int((orbsym == g).sum())
        for j in range(m):
            for i in range(j + 1):
                f[off + i, off + j] = f[off + j, off + i] = d["fock_packed"][k]
                k += 1
        off += m
    eri = np.zeros((n, n, n, n))
    for v, (p, q, r, s) in zip(d["vals"], d["idx"] - 1):
        for a, b, c, e in ((p, q, r, s), (q, p, r, s), (p, q, s, r), (q, p, s, r),
                           (r, s, p, q), (s, r, p, q), (r, s, q, p), (s, r, q, p)):
            eri[a, b, c, e] = v
    o = ref["orbitals"]
    sp = hm.OrbitalSpace(orbsym, o["occ"], o["frozen"], o["deleted"])
    return hm.DenseIntegrals(sp, f, eri), float(d["eref"]), ref


def test_fixture_fock_is_the_scf_one():
    ints, eref, ref = ch2_dz_integrals()
    d = np.load(os.path.join(GOLD, "ch2_dz_dalton.npz"))
    # canonical SCF orbitals: the Fock matrix is diagonal with the orbital energies
    assert np.abs(ints.f - np.diag(np.diag(ints.f))).max() < 1e-8
    assert np.abs(np.diag(ints.f) - d["orb_en"]).max() < 1e-10
    assert abs(eref - ref["history"][0][1]) < 1e-11


def test_ccsdt_iterations_match_the_reference():
    ints, eref, ref = ch2_dz_integrals()
    s = cc.CCSolver(OracleEngine(route=3), ints, method="ccsdt")
    s.load_hamiltonian()
    e = s.solve(maxiter=40, conv=1e-10)
    assert len(s.history) == len(ref["history"]) == 22
    for (i, en, rn), (j, er, rr) in zip(s.history, ref["history"]):
        assert i == j
        assert abs(eref + en - er) < 1e-11, (i, eref + en, er)   # 12 decimals printed
        assert rn == pytest.approx(rr, rel=6e-4), (i, rn, rr)    # 4 digits printed
    assert abs(eref + e - ref["final_energy"]) < 1e-11


def test_ccsd_iterations_match_the_reference():
    # the CCSD ground state of test/CC-excite-I.e.ref on the same integrals
    # (frozen core, nothing deleted), through the CCSD formula: the 16
    # iterations the reference printed, energies to 12 decimals
    ints, eref, _ = ch2_dz_integrals()
    ref = json.load(open(os.path.join(GOLD, "ch2_dz_ccsd_ref.json")))
    o = ref["orbitals"]
    sp = hm.OrbitalSpace(ints.space.orbsym, o["occ"], o["frozen"], o["deleted"])
    s = cc.CCSolver(OracleEngine(route=3), hm.DenseIntegrals(sp, ints.f, ints.eri),
                    method="ccsd")
    s.load_hamiltonian()
    n = len(ref["history"])
    s.solve(maxiter=n, conv=0.0)
    assert n == 16 and len(s.history) == n
    for (i, en, rn), (j, er, rr) in zip(s.history, ref["history"]):
        assert i == j
        assert abs(eref + en - er) < 1e-11, (i, eref + en, er)
        assert rn == pytest.approx(rr, rel=6e-4), (i, rn, rr)
    assert abs(eref + s.history[-1][1] - ref["final_energy"]) < 1e-11
