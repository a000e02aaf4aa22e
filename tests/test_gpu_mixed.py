"""Mixed-precision CCSD (split-TF32 tensor-core contractions until the
residual is small, FP64 after that) converges to the same energy as the
plain FP64 solve, to far below 1 uEh, on a size where the particle ladder
does run on the tensor cores."""
import pytest

import cc
import gccu
import hamiltonian as hm
from devfill import TorchIntegrals

pytestmark = pytest.mark.gpu


def _solve(mixed):
    sp, eps, B = hm.synthetic(6, 30, 60, seed=6030)
    e = gccu.Engine(0)
    try:
        s = cc.CCSolver(e, hm.FactorizedIntegrals(sp, eps, B), method="ccsd")
        s.load_hamiltonian_device(TorchIntegrals(sp, eps, B))
        if mixed:
            en = s.solve_mixed(maxiter=60, conv=1e-9, switch=1e-5)
        else:
            en = s.solve(maxiter=60, conv=1e-9, use_graph=True)
        return en, s.history[-1][2]
    finally:
        e.close()


def test_mixed_solve_reaches_fp64_energy(built):
    e64, r64 = _solve(False)
    emx, rmx = _solve(True)
    assert r64 < 1e-8 and rmx < 1e-8
    assert abs(emx - e64) < 1e-8
