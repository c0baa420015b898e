"""The multi-GPU path is replicas only (every rank advances its own grid, no
data-path collective); its host logic -- the max-over-ranks timing and the
whole-job rate -- runs here as two gloo ranks on the CPU."""
import os
import socket

import pytest

torch = pytest.importorskip("torch")
import torch.distributed as dist  # noqa: E402
import torch.multiprocessing as mp  # noqa: E402


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank_main(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import datetime
    import bench
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        mine = [0.25, 0.75][rank]
        t = bench.max_over_ranks(mine, world, "cpu")
        rate = bench.whole_job_rate(1000, 10, t, world)
        out[rank] = (t, rate)
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_and_whole_job_rate_two_gloo_ranks():
    world = 2
    port = _free_port()
    ctx = mp.get_context("spawn")
    out = ctx.Manager().dict()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, out)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    for r in range(world):
        t, rate = out[r]
        assert t == 0.75                          # the slowest rank
        assert rate == pytest.approx(2 * 1000 * 10 / 0.75)


def test_single_rank_is_the_identity():
    import bench
    assert bench.max_over_ranks(1.5, 1) == 1.5
    assert bench.whole_job_rate(4, 3, 2.0, 1) == 6.0
