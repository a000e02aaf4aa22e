"""The engine's share of a sharded evaluation (gccu_set_shard), on one GPU:
the ranks' shares of one CCSD evaluation are run one after another in one
process (no rank waits for another), and the sum of their residual and
energy lists equals the unsharded evaluation, in FP64, split TF32 and four
int8 slices, for two and three ranks."""
import numpy as np
import pytest

import cc
import gccu
import hamiltonian as hm
from devfill import TorchIntegrals

pytestmark = pytest.mark.gpu


class _Rank:
    def __init__(self, rank, n):
        self.rank, self.n = rank, n


@pytest.mark.parametrize("mode", [0, 1, 3], ids=["fp64", "split_tf32", "int8_slices"])
def test_shares_sum_to_the_whole_evaluation(built, mode):
    sp, eps, B = hm.synthetic(6, 30, 60, seed=6030)
    e = gccu.Engine(0)
    try:
        s = cc.CCSolver(e, hm.FactorizedIntegrals(sp, eps, B), method="ccsd")
        s.load_hamiltonian_device(TorchIntegrals(sp, eps, B))
        for _ in range(2):  # nonzero amplitudes
            s.iterate()
            s.step()
        e.set_precision(mode)
        names = [n for n in cc.Shard.LISTS if n in s.lists]
        s.evaluate()
        whole = {n: e.download(s.lid(n), s.lists[n][1]) for n in names}
        for nranks in (2, 3):
            acc = {n: np.zeros_like(x) for n, x in whole.items()}
            for rank in range(nranks):
                s.shard = _Rank(rank, nranks)
                s.evaluate()
                for n in names:
                    acc[n] += e.download(s.lid(n), s.lists[n][1])
            s.shard = None
            for n in names:
                scale = max(1.0, np.abs(whole[n]).max())
                assert np.max(np.abs(acc[n] - whole[n])) <= 1e-12 * scale, (n, nranks)
    finally:
        e.close()
