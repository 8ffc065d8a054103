"""The N > 1 path of bench.py on CPU: two gloo ranks agree on the slowest
rank's time and on the whole-job rate (weak scaling: every rank's sites
over the slowest rank's time)."""
import os
import socket

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _rank(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    import bench

    my_ms = 10.0 + 5.0 * rank
    m = bench.max_over_ranks(dist, my_ms, None)
    rate = bench.whole_job_rate(world, 1000, 7, m)
    q.put((rank, m, rate))
    dist.barrier()
    dist.destroy_process_group()


@pytest.mark.parametrize("world", [2])
def test_two_gloo_ranks_aggregate(world):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    out = [q.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    slowest = 10.0 + 5.0 * (world - 1)
    for rank, m, rate in out:
        assert m == slowest
        assert rate == pytest.approx(1000 * world * 7 / (slowest * 1e6))
