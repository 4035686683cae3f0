"""Replica plumbing of the multi-GPU bench (ranks.py) on two gloo ranks: the barrier, the
maximum of per-rank durations seen by every rank, and the whole-job rate from it."""
import multiprocessing as mp
import socket
from datetime import timedelta

import pytest

import ranks


def _rank(rank, world, port, q):
    import torch.distributed as dist
    dist.init_process_group('gloo', init_method=f'tcp://127.0.0.1:{port}', rank=rank, world_size=world,
                            timeout=timedelta(seconds=60))
    ranks.barrier()
    slowest = ranks.max_over_ranks(1.0 + rank)   # rank r took 1 + r seconds
    rate = ranks.whole_job_rate(100, slowest)
    q.put((rank, ranks.world_size(), slowest, rate))
    dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(('127.0.0.1', 0))
        return s.getsockname()[1]


def test_single_process_is_identity():
    assert ranks.world_size() == 1
    assert ranks.max_over_ranks(2.5) == 2.5
    assert ranks.whole_job_rate(10, 2.0) == 5.0


def test_two_gloo_ranks_agree_on_the_slowest():
    ctx = mp.get_context('spawn')
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for r, (rank, world, slowest, rate) in enumerate(got):
        assert (rank, world, slowest) == (r, 2, 2.0)
        assert rate == pytest.approx(2 * 100 / 2.0)
