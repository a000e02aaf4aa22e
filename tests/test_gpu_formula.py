"""The formula executor on the device (gccu_formula_run): the CCSD formula
as one engine item list, its intermediates created and deleted by [NEW] /
[DEL] items inside one arena, gives the iterates of the host-driven
evaluation (eagerly and replayed from a CUDA graph, with the residuals'
singlet projection as a target step); the targets' values (frm_sched2's
xret) are the residual norms and the energy; the reference's MP2 run."""
import json
import os

import numpy as np
import pytest

import cc
import gccu
import hamiltonian as hm
from devfill import TorchIntegrals

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(__file__), "golden")


def _solve(native, use_graph, spin_project=False):
    sp, eps, B = hm.synthetic(6, 30, 60, seed=6030)
    e = gccu.Engine(0)
    try:
        s = cc.CCSolver(e, hm.FactorizedIntegrals(sp, eps, B), method="ccsd",
                        native_formula=native, spin_project=spin_project)
        s.load_hamiltonian_device(TorchIntegrals(sp, eps, B))
        s.solve(maxiter=30, conv=1e-9, use_graph=use_graph)
        info = e.formula_info(s.fid) if native else None
        return s.history, info
    finally:
        e.close()


@pytest.mark.parametrize("use_graph", [False, True], ids=["eager", "graph"])
def test_native_ccsd_formula_follows_the_host_loop(built, use_graph):
    ref, _ = _solve(False, use_graph)
    got, info = _solve(True, use_graph)
    assert len(got) == len(ref) and got[-1][2] < 1e-9
    for (_, ea, ra), (_, eb, rb) in zip(ref, got):
        assert abs(ea - eb) < 1e-12 and abs(ra - rb) <= 1e-12 * max(1.0, ra)
    assert info["arena_bytes"] < info["sum_bytes"]


def test_native_formula_with_singlet_projection(built):
    ref, _ = _solve(False, True)
    got, _ = _solve(True, True, spin_project=True)
    assert len(got) == len(ref)
    for (_, ea, ra), (_, eb, rb) in zip(ref, got):
        assert abs(ea - eb) < 1e-11 and abs(ra - rb) <= 1e-11 * max(1.0, ra)


def test_formula_target_values(built):
    sp, eps, B = hm.synthetic(4, 12, 30, seed=12)
    e = gccu.Engine(0)
    try:
        s = cc.CCSolver(e, hm.FactorizedIntegrals(sp, eps, B), method="ccsd",
                        native_formula=True)
        s.load_hamiltonian_device(TorchIntegrals(sp, eps, B))
        for _ in range(2):
            s.iterate()
            s.step()
        info = e.formula_info(s.fid)
        xret = e.formula_run(s.fid, info["targets"])
        items = s.formula_items()
        targets = [it.list for it in items if it.command == gccu.CMD_TARGET]
        last = {lid: i for i, lid in enumerate(targets)}
        for name in ("R1", "R2"):
            lid = s.lid(name)
            assert abs(xret[last[lid]] - np.sqrt(e.dot(lid, lid))) <= 1e-12 * xret[last[lid]]
        assert xret[last[s.lid("E")]] == s.energy()
    finally:
        e.close()


def test_native_mp2_formula_gives_the_reference_energy(built):
    d = hm.read_fcidump(os.path.join(GOLD, "hf_ccpvdz_fcidump.npz"))
    sp = hm.OrbitalSpace(d["orbsym"], [3, 1, 1, 0], [1, 0, 0, 0])
    ints = hm.DenseIntegrals(sp, hm.fock(d["h"], d["eri"], sp.occ_all), d["eri"])
    gold = json.load(open(os.path.join(GOLD, "hf_ccpvdz_ref.json")))
    e = gccu.Engine(0)
    try:
        s = cc.CCSolver(e, ints, method="mp2", native_formula=True)
        s.load_hamiltonian()
        en = s.solve(maxiter=5, conv=1e-10, diis=False)
        assert abs(en + gold["lmp2_norm"]) < 1e-12
    finally:
        e.close()
