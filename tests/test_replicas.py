"""Replica timing on N ranks (gloo, world_size 2, CPU): the job time is the
max over ranks, every rank gets the same value, throughput counts all
ranks' units."""
import os
import socket

import pytest
import torch.multiprocessing as mp

from qclab_b200.replicas import job_throughput, job_time_ms, replica_seed


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    from datetime import timedelta
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        local = [12.5, 30.0][rank]
        ms = job_time_ms(local, dist)
        e2e = job_time_ms(float("inf") if rank == 1 else 5.0, dist)
        out[rank] = (ms, job_throughput(100, 4, ms, world), e2e, replica_seed(7, rank))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_job_time_is_max_over_ranks():
    ctx = mp.get_context("spawn")
    with ctx.Manager() as m:
        out = m.dict()
        mp.start_processes(_rank_main, args=(2, _free_port(), out), nprocs=2, join=True,
                           start_method="spawn")
        res = dict(out)
    assert res[0][0] == res[1][0] == 30.0
    assert res[0][1] == pytest.approx(2 * 100 * 4 / 0.030)
    assert res[0][2] == res[1][2] == float("inf")   # a failed rank poisons the e2e time
    assert {res[0][3], res[1][3]} == {7, 8}


def test_single_process_paths():
    assert job_time_ms(3.0) == 3.0
    assert job_throughput(10, 2, 1000.0, 1) == 20.0
    with pytest.raises(ValueError):
        job_throughput(10, 2, 0.0, 1)
