"""Replica-parallel host logic on CPU: two gloo ranks, max-over-ranks timing."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, q):
    import torch.distributed as dist
    from oceansar_b200 import replicas
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        seconds = 1.0 + rank          # rank 1 is the slow one
        thr, tmax = replicas.job_throughput(1000.0, seconds)
        q.put((rank, replicas.replica_seed(7, rank), thr, tmax))
    finally:
        dist.destroy_process_group()


def test_two_rank_replicas():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [o[1] for o in out] == [7, 8]
    for _, _, thr, tmax in out:
        assert tmax == pytest.approx(2.0)
        assert thr == pytest.approx(2 * 1000.0 / 2.0)


def test_single_process_no_group():
    from oceansar_b200 import replicas
    assert replicas.max_over_ranks(3.5) == 3.5
    assert replicas.job_throughput(10.0, 2.0) == (5.0, 2.0)
