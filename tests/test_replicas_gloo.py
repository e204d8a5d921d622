"""Multi-GPU bookkeeping of bench.py on CPU: two gloo ranks take the MAX of their
device-timed durations and report the whole-job rate from it (replicas, no
data-path collective)."""
import os
import socket

import pytest
import torch.multiprocessing as mp

from hdrestir_b200 import replicas


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, local_ms, out):
    import datetime

    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        r, lr, w = replicas.dist_env()
        replicas.barrier(w, cuda=False)
        m = replicas.max_over_ranks(local_ms[rank], w, device="cpu")
        rate = replicas.whole_job_rate(10, w, m)
        replicas.barrier(w, cuda=False)
        out.put((r, lr, w, m, rate))
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_and_whole_job_rate_two_ranks():
    world = 2
    local_ms = [400.0, 500.0]  # rank 1 is the slower replica
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, world, port, local_ms, q)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    got = sorted(q.get(timeout=10) for _ in range(world))
    for r, (rank, local_rank, w, m, rate) in enumerate(got):
        assert (rank, local_rank, w) == (r, r, world)
        assert m == 500.0  # every rank sees the slowest rank's time
        assert rate == pytest.approx(world * 10 / 0.5)  # 2 replicas x 10 frames in 0.5 s


def test_single_rank_is_identity():
    assert replicas.max_over_ranks(12.5, 1) == 12.5
    assert replicas.whole_job_rate(20, 1, 1000.0) == pytest.approx(20.0)
    with pytest.raises(ValueError):
        replicas.whole_job_rate(1, 1, 0.0)
