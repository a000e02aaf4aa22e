"""CCSDT (the reference's CC maxexc=3, test/CC-energy-I.inp) and CCSDTQ as
chains of binary contractions (cc.excitation_formula, factors from the Wick
signs of cc.contraction_sign) on the CPU oracle, against <mu| e^-T H e^T |0>
evaluated in the full Fock space of ten spin orbitals with a non-canonical
Fock matrix, so that every term of the formula contributes; a CCSDT solve,
whose converged amplitudes make the Fock-space residuals vanish and whose
energy lies closer to the full CI energy than the CCSD one; the formula on
the product planner, at the CCSDT configuration's size too."""
import numpy as np
import pytest

import cc
import dense_cc
import hamiltonian as hm
from engine import OracleEngine
from fock_cc import FockSpace, non_canonical_fock, random_amplitudes


def _system(no, nv, seed, method="ccsdt", nsym=1):
    sp, eps, B = hm.synthetic(no, nv, 12, seed=seed, nsym=nsym)
    ints = hm.FactorizedIntegrals(sp, eps, B)
    dense = hm.DenseIntegrals(sp, np.diag(eps), ints.dense_eri())
    F, W, nso = dense_cc.spin_orbital(sp, dense.f, dense.eri_elems)
    s = cc.CCSolver(OracleEngine(route=3), ints, method=method)
    s.load_hamiltonian()
    return s, F, W, nso


def _spin_orbital_irreps(s):
    """0-based irrep of every spin orbital (holes, then particles), for the
    direct product as XOR"""
    sp = s.ints.space
    orbs = np.concatenate([sp.hole, sp.part])
    return np.asarray(sp.orbsym)[orbs[np.arange(2 * len(orbs)) // 2]] - 1


def _set_fock(s, F, nso):
    o, v = slice(0, nso), slice(nso, F.shape[0])
    s.freeze_hamiltonian(False)
    s.e.upload(s.lid("F"), s.view("F").from_dense(
        {1: F[o, o], 2: F[o, v], 3: F[v, o], 4: F[v, v]}, s.lists["F"][1]))
    s.freeze_hamiltonian(True)


def _dense(s, name, shape):
    x = s.e.download(s.lid(name), s.lists[name][1])
    return s.view(name).to_dense(x, 1, shape)


def test_terms_and_factors():
    # 48 terms up to doubles (CCSD, the energy included), 102 up to triples;
    # every factor is +-1 over the m! of identical attachments
    from math import factorial
    assert len(cc.excitation_terms(2)) == 48
    assert len(cc.excitation_terms(3)) == 102
    for name, key, steps, _ in cc.excitation_terms(3):
        den = np.prod([factorial(steps.count(st)) for st in set(steps)])
        assert abs(abs(cc.term_factor(name, key, steps)) * den - 1.0) < 1e-15


@pytest.mark.parametrize("no,nv,seed", [(3, 2, 21), (2, 3, 22)])
def test_ccsdt_residuals_match_fock_space(built, no, nv, seed):
    s, F, W, nso = _system(no, nv, seed)
    rng = np.random.default_rng(seed)
    F = non_canonical_fock(F, nso, rng)
    _set_fock(s, F, nso)
    nvo = F.shape[0] - nso
    amps = {r: random_amplitudes(r, nvo, nso, rng) for r in (1, 2, 3)}
    for r, t in amps.items():
        s.e.upload(s.lid(f"T{r}"), s.view(f"T{r}").from_dense({1: t}, s.lists[f"T{r}"][1]))
    s.evaluate()
    ref = FockSpace(F, W, nso).residuals(amps, 3)
    assert abs(s.energy() - ref[0]) < 1e-13
    for r in (1, 2, 3):
        got = _dense(s, f"R{r}", ref[r].shape)
        assert np.abs(ref[r]).max() > 1e-3
        assert np.abs(got - ref[r]).max() < 1e-12 * np.abs(ref[r]).max(), r


def test_ccsdt_solve_zeroes_the_fock_space_residuals():
    s, F, W, nso = _system(2, 2, 23)
    e = s.solve(maxiter=80, conv=1e-11)
    assert s.history[-1][2] < 1e-11
    nvo = F.shape[0] - nso
    amps = {r: _dense(s, f"T{r}", (nvo,) * r + (nso,) * r) for r in (1, 2, 3)}
    assert np.abs(amps[3]).max() > 1e-6
    fs = FockSpace(F, W, nso)
    ref = fs.residuals(amps, 3)
    assert abs(e - ref[0]) < 1e-12
    for r in (1, 2, 3):
        assert np.abs(ref[r]).max() < 1e-9, r
    # full CI in the sector of the reference's electron count
    dim = 1 << fs.n
    sector = [d for d in range(dim) if bin(d).count("1") == nso]
    Hs = fs.H[sector][:, sector].toarray()
    e_fci = np.linalg.eigvalsh(Hs)[0] - fs.H[fs.ref, fs.ref]
    s2, _, _, _ = _system(2, 2, 23, method="ccsd")
    e_ccsd = s2.solve(maxiter=80, conv=1e-11)
    assert abs(e - e_fci) < abs(e_ccsd - e_fci)


def test_ccsdt_formula_plans_on_the_product_engine(built):
    # every [CONTR] of the formula passes the product planner's checks
    # (host-only engine, no device) on a C2v space
    import gccu
    sp, eps, B = hm.synthetic(3, 6, 12, seed=24, nsym=4)
    e = gccu.Engine(-1)
    try:
        s = cc.CCSolver(e, hm.FactorizedIntegrals(sp, eps, B), method="ccsdt")
        nitems = 0
        for it in s.formula:
            if it["kind"] != "CONTR":
                continue
            c = np.asarray(it["cnt"])
            ex1 = np.asarray(it["op1"][1]) - c
            ex2 = np.asarray(it["op2"][1]) - np.concatenate([c[4:], c[:4]])
            n, st = e.plan_info(s.blk(it["op1"]), s.blk(it["op2"]), s.blk(it["res"]), ex1, ex2,
                                c)
            nitems += n
        assert nitems > 0
    finally:
        e.close()


@pytest.mark.parametrize("no,nv,nsym,seed", [(2, 3, 4, 25), (3, 2, 2, 26)])
def test_ccsdt_residuals_with_point_group_symmetry(built, no, nv, nsym, seed):
    # symmetry-blocked lists (irreps round-robin over the orbitals): the
    # formula's residuals equal the Fock-space ones for totally symmetric
    # amplitudes and a totally symmetric non-canonical Fock matrix
    s, F, W, nso = _system(no, nv, seed, nsym=nsym)
    assert s.nsym == nsym
    irr = _spin_orbital_irreps(s)
    rng = np.random.default_rng(seed)
    F = non_canonical_fock(F, nso, rng) * (irr[:, None] == irr[None, :])
    _set_fock(s, F, nso)
    nvo = F.shape[0] - nso
    amps = {}
    for r in (1, 2, 3):
        t = random_amplitudes(r, nvo, nso, rng)
        grids = np.meshgrid(*([irr[nso:]] * r + [irr[:nso]] * r), indexing="ij")
        prod = np.zeros(t.shape, dtype=np.int64)
        for g in grids:
            prod ^= g
        amps[r] = t * (prod == 0)
        s.e.upload(s.lid(f"T{r}"), s.view(f"T{r}").from_dense({1: amps[r]}, s.lists[f"T{r}"][1]))
    s.evaluate()
    ref = FockSpace(F, W, nso).residuals(amps, 3)
    assert abs(s.energy() - ref[0]) < 1e-13
    for r in (1, 2, 3):
        got = _dense(s, f"R{r}", ref[r].shape)
        assert np.abs(ref[r]).max() > 1e-4, r
        assert np.abs(got - ref[r]).max() < 1e-12 * np.abs(ref[r]).max(), r


def test_ccsdt_lists_filled_through_the_device_path(built):
    # the Hamiltonian and the T1..T3 denominators generated by torch (the
    # device fill, here on the CPU) equal the host fill on a space of four
    # irreps, and one evaluation from the same amplitudes agrees
    from devfill import TorchIntegrals
    sp, eps, B = hm.synthetic(3, 6, 12, seed=27, nsym=4)
    ints = hm.FactorizedIntegrals(sp, eps, B)
    host = cc.CCSolver(OracleEngine(route=3), ints, method="ccsdt")
    host.load_hamiltonian()
    dev = cc.CCSolver(OracleEngine(route=3), ints, method="ccsdt")
    dev.load_hamiltonian_device(TorchIntegrals(sp, eps, B, device="cpu"))
    for name in ("F", "V", "DT1", "DT2", "DT3"):
        a, b = host.e.data[host.lid(name)], dev.e.data[dev.lid(name)]
        assert a.size > 0 and np.max(np.abs(a - b)) <= 1e-13 * max(1.0, np.abs(a).max()), name
    for s in (host, dev):
        for r in (1, 2, 3):
            n = s.lists[f"T{r}"][1]
            s.e.upload(s.lid(f"T{r}"), 0.05 * np.random.default_rng(r).standard_normal(n))
        s.evaluate()
    for name in ("R1", "R2", "R3"):
        a, b = host.e.data[host.lid(name)], dev.e.data[dev.lid(name)]
        assert np.max(np.abs(a - b)) <= 1e-12 * np.abs(a).max(), name


def test_ccsdt_plans_at_the_ccsdt_configuration(built):
    # the CCSDT configuration's orbital space (D2h, irreps round-robin,
    # o6/v48): every [CONTR] plans on the product engine (host-only), with
    # hundreds of thousands of uneven block contractions per evaluation
    import gccu
    sp, eps, B = hm.synthetic(6, 48, 8, seed=1001, nsym=8)
    e = gccu.Engine(-1)
    try:
        s = cc.CCSolver(e, hm.FactorizedIntegrals(sp, eps, B), method="ccsdt")
        nitems, flops = 0, 0.0
        for it in s.formula:
            if it["kind"] != "CONTR":
                continue
            c = np.asarray(it["cnt"])
            ex1 = np.asarray(it["op1"][1]) - c
            ex2 = np.asarray(it["op2"][1]) - np.concatenate([c[4:], c[:4]])
            n, st = e.plan_info(s.blk(it["op1"]), s.blk(it["op2"]), s.blk(it["res"]), ex1, ex2,
                                c)
            nitems += n
            flops += st[7]
        assert nitems == 659388
        assert 0.05e12 < flops < 0.2e12
    finally:
        e.close()


@pytest.mark.parametrize("no,nv,seed", [(3, 2, 28), (2, 3, 29)])
def test_ccsdtq_residuals_match_fock_space(built, no, nv, seed):
    # the same generator one excitation level higher: T1..T4, R1..R4
    s, F, W, nso = _system(no, nv, seed, method="ccsdtq")
    rng = np.random.default_rng(seed)
    F = non_canonical_fock(F, nso, rng)
    _set_fock(s, F, nso)
    nvo = F.shape[0] - nso
    amps = {r: random_amplitudes(r, nvo, nso, rng) for r in (1, 2, 3, 4)}
    for r, t in amps.items():
        s.e.upload(s.lid(f"T{r}"), s.view(f"T{r}").from_dense({1: t}, s.lists[f"T{r}"][1]))
    s.evaluate()
    ref = FockSpace(F, W, nso).residuals(amps, 4)
    assert abs(s.energy() - ref[0]) < 1e-13
    for r in (1, 2, 3, 4):
        got = _dense(s, f"R{r}", ref[r].shape)
        assert np.abs(ref[r]).max() > 1e-4, r
        assert np.abs(got - ref[r]).max() < 1e-12 * np.abs(ref[r]).max(), r
