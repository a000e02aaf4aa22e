"""Owner-computes sharding of the CC evaluation over ranks (cc.Shard), on
CPU with two gloo ranks: each rank runs the oracle engine, the residual and
energy contractions compute only that rank's block contractions, the [ADD]s
into them count on rank 0, the intermediates are computed in full, and the
residual and energy lists are summed over the ranks after each evaluation.
Four DIIS iterations give the energies, residual norms and amplitudes of the
unsharded single-process solve."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _system():
    import hamiltonian as hm
    sp, eps, B = hm.synthetic(3, 7, 20, seed=31)
    return hm.FactorizedIntegrals(sp, eps, B)


def _solve(shard):
    import cc
    from engine import OracleEngine
    s = cc.CCSolver(OracleEngine(route=3), _system(), method="ccsd", shard=shard)
    s.load_hamiltonian()
    s.solve(maxiter=4, conv=0.0)
    return s


def _rank(rank, world, port, out):
    import datetime

    import torch.distributed as dist

    import cc

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        s = _solve(cc.Shard(dist))
        out[rank] = (s.history, {a: s.e.data[s.lid(a)].copy() for a in s.amps})
        dist.barrier()
    finally:
        dist.destroy_process_group()


@pytest.mark.timeout(240)
def test_sharded_solve_equals_single_rank(built):
    ref = _solve(None)
    ctx = mp.get_context("spawn")
    with ctx.Manager() as m:
        out = m.dict()
        port = _free_port()
        procs = [ctx.Process(target=_rank, args=(r, 2, port, out)) for r in range(2)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(200)
        assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
        for rank in range(2):
            hist, amps = out[rank]
            for (i, ea, ra), (_, eb, rb) in zip(hist, ref.history):
                assert abs(ea - eb) < 1e-12 and abs(ra - rb) < 1e-12 * max(1.0, rb), (rank, i)
            for a, x in amps.items():
                y = ref.e.data[ref.lid(a)]
                assert np.max(np.abs(x - y)) <= 1e-12 * max(1.0, np.abs(y).max()), (rank, a)
