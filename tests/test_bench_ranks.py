"""bench.py's multi-process timing on CPU: with two gloo ranks (the process
layout of `bench.py --gpus 2` under torchrun, one process per device), every
rank ends up with the slowest rank's time, and without a process group the
time is returned unchanged."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, values, out):
    import datetime

    import torch.distributed as dist

    import bench

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        out[rank] = bench.max_over_ranks(values[rank], dist)
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_without_group():
    import bench

    assert bench.max_over_ranks(3.5, None) == 3.5


@pytest.mark.timeout(180)
def test_max_over_two_gloo_ranks():
    ctx = mp.get_context("spawn")
    with ctx.Manager() as m:
        out = m.dict()
        values = [12.5, 17.25]
        port = _free_port()
        procs = [ctx.Process(target=_rank, args=(r, 2, port, values, out)) for r in range(2)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(150)
        assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
        assert dict(out) == {0: 17.25, 1: 17.25}
