"""The N > 1 path of bench.py on the CPU: two gloo ranks, each with its own
operand seeds, timing reduced to the slowest rank, whole-job rate from it."""
import os
import socket

import pytest
import torch.multiprocessing as mp

from libfastlib_b200.replicas import max_over_ranks, operand_seeds, whole_job_rate


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    import torch.distributed as dist
    from datetime import timedelta
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        local_ms = [12.5, 17.25][rank]
        ms = max_over_ranks(local_ms)
        out[rank] = (ms, whole_job_rate(1000, 4, ms, world), operand_seeds(rank, 5))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks():
    world, port = 2, _free_port()
    with mp.Manager() as m:
        out = m.dict()
        mp.spawn(_rank, args=(world, port, out), nprocs=world, join=True)
        res = dict(out)
    for r in range(world):
        ms, rate, seeds = res[r]
        assert ms == 17.25                       # the slowest rank's time on every rank
        assert rate == pytest.approx(world * 1000 * 4 / (17.25 / 1e3) / 1e9)
    s0, s1 = {x for p in res[0][2] for x in p}, {x for p in res[1][2] for x in p}
    assert len(s0) == 10 and not (s0 & s1)       # ranks build disjoint operand pairs


def test_single_process_is_identity():
    assert max_over_ranks(3.5) == 3.5
    assert whole_job_rate(2_000_000, 10, 4.0, 1) == pytest.approx(5.0)
