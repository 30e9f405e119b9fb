"""The multi-GPU bench path is replicas: every rank solves its own copy, and
the job's time is the slowest rank's (max over ranks), its throughput all
ranks' texels over that time.  Checked here with two gloo ranks on the CPU."""
import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank: int, world: int, port: int, out):
    import datetime

    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        local_ms = [12.5, 20.0][rank]
        ms = bench.max_over_ranks(local_ms, dist, device="cpu")
        out.put((rank, ms, bench.job_rate(world, 3e6, ms)))
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_and_job_rate():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    res = sorted(q.get(timeout=10) for _ in range(2))
    for _, ms, rate in res:
        assert ms == 20.0  # the slowest rank
        assert rate == pytest.approx(2 * 3e6 / 20e-3 / 1e6)


def test_single_rank_is_unchanged():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.max_over_ranks(7.0, None) == 7.0
    assert bench.job_rate(1, 1e6, 1000.0) == pytest.approx(1.0)
