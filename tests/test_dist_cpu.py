"""Multi-rank plumbing of bench.py on CPU: two gloo ranks run the barrier and
the max / sum reductions used to time N independent replicas (one per GPU)."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank_main(rank, world, port, out):
    import datetime

    import torch.distributed as dist

    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        bench.barrier(world)
        # rank r took (r + 1) * 10 ms for (r + 1) * 1000 keys
        out[rank] = (bench.max_over_ranks((rank + 1) * 10.0, world),
                     bench.sum_over_ranks((rank + 1) * 1000.0, world))
        bench.barrier(world)
    finally:
        dist.destroy_process_group()


@pytest.mark.timeout(120)
def test_two_rank_replica_timing_reductions():
    ctx = mp.get_context("spawn")
    world = 2
    manager = ctx.Manager()
    out = manager.dict()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, out)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(90)
        assert p.exitcode == 0
    # every rank sees the slowest rank's time and the total work
    assert out[0] == out[1] == (20.0, 3000.0)
