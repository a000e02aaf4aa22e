"""CC drivers on the GPU engine: the reference's golden MP2 run, CCSD against
the dense spin-orbital CCSD and the CPU oracle, CUDA-graph replay, device-side
Hamiltonian generation."""
import json
import os

import numpy as np
import pytest

import cc
import dense_cc
import gccu
import hamiltonian as hm
from engine import OracleEngine

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(__file__), "golden")


@pytest.fixture(scope="module")
def hf_ints():
    d = hm.read_fcidump(os.path.join(GOLD, "hf_ccpvdz_fcidump.npz"))
    sp = hm.OrbitalSpace(d["orbsym"], [3, 1, 1, 0], [1, 0, 0, 0])
    f = hm.fock(d["h"], d["eri"], sp.occ_all)
    return hm.DenseIntegrals(sp, f, d["eri"])


@pytest.fixture
def engine(built):
    e = gccu.Engine(0)
    yield e
    e.close()


def test_mp2_golden_on_gpu(engine, hf_ints):
    gold = json.load(open(os.path.join(GOLD, "hf_ccpvdz_ref.json")))
    s = cc.CCSolver(engine, hf_ints, method="mp2")
    s.load_hamiltonian()
    e = s.solve(maxiter=5, conv=1e-10, diis=False)
    (_, e1, r1), (_, e2, r2) = s.history[:2]
    assert e1 == 0.0 and round(r1, 3) == 1.100
    assert abs(e + gold["lmp2_norm"]) < 1e-12
    assert abs(e2 - gold["final_energy_12digits"]) < 1e-12
    assert r2 < 1e-12


def test_ccsd_matches_dense_and_oracle(engine, hf_ints):
    F, W, no = dense_cc.spin_orbital(hf_ints.space, hf_ints.f, hf_ints.eri_elems)
    _, hd = dense_cc.ccsd(F, W, no, maxiter=6)
    s = cc.CCSolver(engine, hf_ints, method="ccsd")
    s.load_hamiltonian()
    s.solve(maxiter=6, conv=1e-14, diis=False)
    for (i, ed, rd), (j, eg, rg) in zip(hd, s.history):
        assert abs(ed - eg) < 1e-11 and abs(rd - rg) < 1e-10 * max(1.0, rd), (i, ed, eg, rd, rg)
    # the same DIIS iterations on the oracle give the same lists
    o = cc.CCSolver(OracleEngine(route=3), hf_ints, method="ccsd")
    o.load_hamiltonian()
    s2 = cc.CCSolver  # noqa: F841
    o.solve(maxiter=4, conv=1e-14, diis=True)
    engine.close()
    e2 = gccu.Engine(0)
    try:
        g = cc.CCSolver(e2, hf_ints, method="ccsd")
        g.load_hamiltonian()
        g.solve(maxiter=4, conv=1e-14, diis=True)
        for name in ("T1", "T2", "R2", "TAU", "XWT"):
            n = g.lists[name][1]
            a = e2.download(g.lid(name), n)
            b = o.e.data[o.lid(name)]
            assert np.max(np.abs(a - b)) <= 1e-11 * max(1.0, np.abs(b).max()), name
    finally:
        e2.close()


def test_graph_replay_same_iterates(engine, hf_ints):
    s = cc.CCSolver(engine, hf_ints, method="ccsd")
    s.load_hamiltonian()
    s.solve(maxiter=6, conv=1e-14, diis=True, use_graph=True)
    assert s.graph is not None
    o = cc.CCSolver(OracleEngine(route=3), hf_ints, method="ccsd")
    o.load_hamiltonian()
    o.solve(maxiter=6, conv=1e-14, diis=True)
    for (i, ea, ra), (j, eb, rb) in zip(s.history, o.history):
        assert abs(ea - eb) < 1e-11 and abs(ra - rb) < 1e-10 * max(1.0, rb)


def test_device_fill_matches_host_fill(engine):
    from devfill import TorchIntegrals
    sp, eps, B = hm.synthetic(4, 9, 30, seed=5, nsym=2)
    ints = hm.FactorizedIntegrals(sp, eps, B)
    s = cc.CCSolver(engine, ints, method="ccsd")
    s.load_hamiltonian_device(TorchIntegrals(sp, eps, B))
    xf, xv = cc.fill_hamiltonian(s.view("F"), s.view("V"), s.lists["F"][1], s.lists["V"][1], ints)
    assert np.allclose(engine.download(s.lid("F"), s.lists["F"][1]), xf, rtol=0, atol=1e-13)
    assert np.allclose(engine.download(s.lid("V"), s.lists["V"][1]), xv, rtol=0, atol=1e-13)
    d2 = cc.fill_denominators(s.view("DT2"), s.lists["T2"][1], s.lists["T2"][2][0], ints)
    assert np.allclose(engine.download(s.lid("DT2"), s.lists["T2"][1]), d2, atol=1e-13)


@pytest.mark.parametrize("mode", [0, 1], ids=["fp64", "split_tf32"])
def test_ccsd_spin_flip_symmetry_same_iterates(built, mode):
    # the engine under use_tr (half of the Ms cases, doubled, sym_ab_blk) gives
    # the iterates of the plain evaluation, replayed from CUDA graphs, on a
    # synthetic system whose particle ladder reaches the tensor cores
    from devfill import TorchIntegrals
    sp, eps, B = hm.synthetic(6, 30, 60, seed=6030)
    hist = []
    for use_tr in (False, True):
        e = gccu.Engine(0)
        try:
            e.set_precision(mode)
            s = cc.CCSolver(e, hm.FactorizedIntegrals(sp, eps, B), method="ccsd", use_tr=use_tr)
            s.load_hamiltonian_device(TorchIntegrals(sp, eps, B))
            s.solve(maxiter=8, conv=1e-14, use_graph=True)
            hist.append(s.history)
        finally:
            e.close()
    tol = 1e-10 if mode == 0 else 1e-6
    for (i, ea, ra), (_, eb, rb) in zip(*hist):
        assert abs(ea - eb) < tol * max(1.0, abs(ea)), (i, ea, eb)
        assert abs(ra - rb) < tol * max(1.0, ra), (i, ra, rb)


def test_fcidump_filled_on_the_device_gives_the_reference_mp2(engine):
    # the FCIDUMP's records scattered into h and (pq|rs) in device memory,
    # the Fock matrix and the lists formed there: the lists of the host fill
    # and the reference's MP2 energy
    from devfill import TorchDenseIntegrals, list_tensor
    path = os.path.join(GOLD, "hf_ccpvdz_fcidump.npz")
    gold = json.load(open(os.path.join(GOLD, "hf_ccpvdz_ref.json")))
    tints = TorchDenseIntegrals.from_fcidump(path, [3, 1, 1, 0], [1, 0, 0, 0])
    s = cc.CCSolver(engine, tints, method="mp2")
    s.load_hamiltonian_device(tints)
    host = cc.CCSolver(OracleEngine(route=3), hm.DenseIntegrals(
        tints.space, tints.f.cpu().numpy(), tints.eri_pqrs.cpu().numpy()), method="mp2")
    host.load_hamiltonian()
    for name in ("F", "V", "DT2"):
        lid, n, _ = s.lists[name]
        got = list_tensor(engine, lid, n).cpu().numpy()
        ref = host.e.data[host.lid(name)]
        assert np.max(np.abs(got - ref)) <= 1e-13 * max(1.0, np.abs(ref).max()), name
    e = s.solve(maxiter=5, conv=1e-10)
    assert abs(e + gold["lmp2_norm"]) < 1e-13
