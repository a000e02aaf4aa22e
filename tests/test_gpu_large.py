"""Parity at the shapes the benchmark runs, against the oracle.

1. Contractions over more than 4096 contraction indices (6 holes, 72
   particles: 5184 particle pairs contracted).  In split TF32 each tile
   accumulates at most 4096 indices in FP32 and the chunks are summed in
   FP64 through the atomic epilogue; the column operand of the first
   contraction has 432 columns, split into two 224-wide tiles, so 128-row
   chunks of the split pre-pass straddle two column bands; the second
   contraction gathers a map-addressed operand (three particle annihilators
   merged from an external and two contracted ones) inside the split
   pre-pass.  In FP64 the same items are split along the contraction index
   across CTAs (atomic epilogue).  Split TF32 at 2e-5, FP64 at 1e-12,
   relative to the largest result element.
2. One whole CCSD formula evaluation at o8/v32/naux160 (the o8/v32 workload
   of the benchmark family) from identical amplitudes: every list the
   evaluation writes (energy, residuals, intermediates) against the oracle
   engine (route 3, OpenBLAS dgemm), per ME-list distribution block, in FP64
   at 1e-12 relative (2-norm of the difference over the block's 2-norm) and
   in split TF32 at 2e-5.
3. The first three FP64 iterations at o12/v100/naux450 (the benchmark
   family's distribution, whose CC iteration diverges at this size) give
   the oracle's energies to 1e-10 Eh and residual norms to 1e-10 relative:
   the divergence is the Hamiltonian's, not the engine's.
"""
import numpy as np
import pytest

import cc
import gccu
import hamiltonian as hm
from binding import Oracle
from cases import H, P, _bc, occ8, random_list
from devfill import TorchIntegrals
from engine import OracleEngine

pytestmark = pytest.mark.gpu

RTOL_TC = 2e-5
RTOL_FP64 = 1e-12

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


@pytest.mark.parametrize("case", BIG_K, ids=[c[0] for c in BIG_K])
def test_contraction_longer_than_one_fp32_chunk(engine, case):
    nsym, norb = BIG_SPACE
    engine.register_orbinfo(nsym, norb)
    o = Oracle(nsym, norb)
    ls = []
    for occ in case[1:4]:
        le, n = engine.register_list(engine.define_operator([occ]))
        lo, _ = o.define_list(o.define_op([occ]))
        ls.append((le, lo, n))
    (l1, o1, n1), (l2, o2, n2), (l12, o12, n12) = ls
    x1, x2 = random_list(n1, 71), random_list(n2, 72)
    x12 = random_list(n12, 73)
    engine.upload(l1, x1)
    engine.upload(l2, x2)
    args = ((l1, 1), (l2, 1), (l12, 1), case[4], case[5], case[6])
    rows = engine.plan_items(*args)
    assert rows[:, 2].max() > 4096  # several FP32 accumulation chunks
    assert (rows[:, 0] > 32).any() and (rows[:, 1] > 32).any()
    ref = x12.copy()
    o.contract(2, o1, 1, x1, o2, 1, x2, o12, 1, ref, case[4], case[5], case[6], -0.5,
               update=True)
    scale = max(1.0, np.abs(ref).max())
    got = {}
    try:
        for mode, tol in ((1, RTOL_TC), (0, RTOL_FP64)):
            engine.set_precision(mode)
            engine.upload(l12, x12)
            engine.contract(*args, fact=-0.5, update=True)
            got[mode] = engine.download(l12, n12)
            err = np.max(np.abs(got[mode] - ref)) / scale
            assert err <= tol, (case[0], mode, err)
    finally:
        engine.set_precision(0)
    # the split-TF32 result is not the FP64 one: the tensor cores ran
    assert np.max(np.abs(got[1] - got[0])) / scale > 1e-10


C0 = dict(nocc=8, nvir=32, naux=160, seed=1000)


def _block_errors(eng, lid, a, b):
    """per distribution block of a list: ||a - b|| / ||b|| (blocks whose norm
    is below 1e-10 of the list's are compared against the list's norm)"""
    tot = max(np.linalg.norm(b), 1e-300)
    worst = 0.0
    for r in eng.dists(lid):
        off, ln = int(r[4]), int(r[5])
        if ln == 0:
            continue
        d = np.linalg.norm(a[off:off + ln] - b[off:off + ln])
        nb = np.linalg.norm(b[off:off + ln])
        worst = max(worst, d / (nb if nb > 1e-10 * tot else tot))
    return worst


@pytest.mark.parametrize("mode,tol", [(0, RTOL_FP64), (1, RTOL_TC)], ids=["fp64", "split_tf32"])
def test_ccsd_evaluation_c0_every_list(engine, mode, tol):
    sp, eps, B = hm.synthetic(C0["nocc"], C0["nvir"], C0["naux"], seed=C0["seed"])
    ints = hm.FactorizedIntegrals(sp, eps, B)
    g = cc.CCSolver(engine, ints, method="ccsd")
    g.load_hamiltonian_device(TorchIntegrals(sp, eps, B))
    for _ in range(2):  # nonzero T1 and T2: two FP64 Jacobi iterations from zero
        g.iterate()
        g.step()
    o = cc.CCSolver(OracleEngine(route=3), ints, method="ccsd")
    for name in ("F", "V", "T1", "T2", "DT1", "DT2"):
        lid, n, _ = g.lists[name]
        o.e.data[o.lid(name)][:] = engine.download(lid, n)
    engine.set_precision(mode)
    try:
        g.evaluate()
        engine.sync()
    finally:
        engine.set_precision(0)
    o.evaluate()
    written = {it["res"][0] for it in cc.CCSD_FORMULA}
    assert len(written) >= 12
    for name in sorted(written):
        lid, n, _ = g.lists[name]
        a = engine.download(lid, n)
        b = o.e.data[o.lid(name)]
        err = _block_errors(engine, lid, a, b)
        assert err <= tol, (name, mode, err)


def test_first_iterations_o12v100_match_oracle(engine):
    import os

    import binding
    binding.set_blas(os.cpu_count())  # route-3 dgemm through OpenBLAS on all host cores
    sp, eps, B = hm.synthetic(12, 100, 450, seed=1010)
    ints = hm.FactorizedIntegrals(sp, eps, B)
    g = cc.CCSolver(engine, ints, method="ccsd")
    g.load_hamiltonian_device(TorchIntegrals(sp, eps, B))
    o = cc.CCSolver(OracleEngine(route=3), ints, method="ccsd")
    for name in ("F", "V", "DT1", "DT2"):
        lid, n, _ = g.lists[name]
        o.e.data[o.lid(name)][:] = engine.download(lid, n)
    g.solve(maxiter=3, conv=0.0, diis=True)
    o.solve(maxiter=3, conv=0.0, diis=True)
    assert len(g.history) == len(o.history) == 3
    for (i, eg, rg), (_, eo, ro) in zip(g.history, o.history):
        assert abs(eg - eo) < 1e-10, (i, eg, eo)
        assert abs(rg - ro) <= 1e-10 * max(1.0, ro), (i, rg, ro)
