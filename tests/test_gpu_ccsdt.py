"""CCSDT on the device: one evaluation of the CCSDT formula
(cc.excitation_formula, 102 terms, three-body amplitudes and intermediates of
up to eight indices) through the engine in FP64 equals the oracle's on the
same amplitudes, in C2v symmetry."""
import numpy as np
import pytest

import cc
import gccu
import hamiltonian as hm
from engine import OracleEngine

pytestmark = pytest.mark.gpu

RTOL = 1e-12


def test_ccsdt_evaluation_matches_oracle(built):
    sp, eps, B = hm.synthetic(3, 6, 12, seed=24, nsym=4)
    ints = hm.FactorizedIntegrals(sp, eps, B)
    out = []
    for eng in (gccu.Engine(0), OracleEngine(route=3)):
        try:
            s = cc.CCSolver(eng, ints, method="ccsdt")
            s.load_hamiltonian()
            for r in (1, 2, 3):
                n = s.lists[f"T{r}"][1]
                s.e.upload(s.lid(f"T{r}"), 0.05 * np.random.default_rng(r).standard_normal(n))
            s.evaluate()
            out.append([np.array([s.energy()])] +
                       [s.e.download(s.lid(f"R{r}"), s.lists[f"R{r}"][1]) for r in (1, 2, 3)])
        finally:
            eng.close()
    for k, (got, ref) in enumerate(zip(*out)):
        assert np.abs(ref).max() > 0, k
        assert np.abs(got - ref).max() <= RTOL * np.abs(ref).max(), k
