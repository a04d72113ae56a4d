"""Multi-rank host logic of bench.py on CPU (gloo, world size 2): every rank runs
its own replica and the reported time is the maximum over ranks."""
import os
import socket

import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, out):
    import datetime

    import torch.distributed as dist

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    import bench

    got = bench.max_over_ranks([10.0 * (rank + 1), 3.0 - rank], dist)
    r, w, _ = bench._dist_env()
    out[rank] = (got, r, w)
    dist.barrier()
    dist.destroy_process_group()


def test_max_over_ranks_gloo_world2():
    ctx = mp.get_context("spawn")
    mgr = ctx.Manager()
    out = mgr.dict()
    port = _free_port()
    mp.start_processes(_worker, args=(2, port, out), nprocs=2, join=True, start_method="spawn")
    for rank in (0, 1):
        got, r, w = out[rank]
        assert got == [20.0, 3.0]
        assert (r, w) == (rank, 2)
