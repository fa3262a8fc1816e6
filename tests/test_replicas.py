"""Multi-process (gloo, world size 2, CPU) tests of the replica bookkeeping
bench.py uses under torchrun: the job time is the slowest rank's and the job
value counts every rank's queries."""
import os
import socket

import pytest
import torch.multiprocessing as mp

from harmonia_b200 import replicas


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, results):
    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=__import__("datetime").timedelta(seconds=60))
    try:
        ms = [1.5, 4.25][rank]
        got = replicas.max_over_ranks(ms)
        seeds = [None] * world
        dist.all_gather_object(seeds, replicas.query_seed(2, rank))
        results[rank] = (got, seeds)
    finally:
        dist.destroy_process_group()


def test_max_over_two_gloo_ranks():
    ctx = mp.get_context("spawn")
    mgr = ctx.Manager()
    results = mgr.dict()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, results)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    assert results[0][0] == results[1][0] == 4.25
    assert len(set(results[0][1])) == 2  # replicas search different batches


def test_job_throughput_counts_all_ranks():
    assert replicas.job_throughput(1 << 24, 4, 1.0) == pytest.approx(4 * (1 << 24) / 1e3)
    assert replicas.max_over_ranks(3.0) == 3.0  # no process group: identity
