"""The multi-GPU path of bench.py is replicas only: every rank runs its own
walkers, and the one cross-rank step is the max-over-ranks time behind the
whole-job rate.  Checked here with two gloo ranks on the CPU."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(('127.0.0.1', 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR='127.0.0.1', MASTER_PORT=str(port))
    dist.init_process_group('gloo', rank=rank, world_size=world)
    try:
        import bench
        # rank r moved 1000 electrons in (1 + r) seconds
        rate, tmax = bench.job_rate(1000, 1.0 + rank, world)
        out[rank] = (rate, tmax)
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_job_rate_takes_the_slowest_rank():
    world = 2
    port = _free_port()
    with mp.get_context('spawn').Manager() as m:
        out = m.dict()
        mp.spawn(_rank, args=(world, port, out), nprocs=world, join=True)
        res = dict(out)
    for r in range(world):
        rate, tmax = res[r]
        assert tmax == 2.0
        assert rate == pytest.approx(1000 * world / 2.0)


def test_job_rate_single_rank():
    import bench
    assert bench.job_rate(500, 0.5, 1) == (1000.0, 0.5)
