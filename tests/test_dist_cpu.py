"""CPU, world_size 2 over gloo: the replica benchmark's multi-rank logic —
per-rank source selection and max/sum aggregation — without a GPU."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp


def _free_port() -> int:
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _rank_main(rank, world, port, q):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    import bench
    d = bench.Dist(world, "cpu")
    deg = np.array([0, 3, 1, 0, 2, 5, 0, 4] * 20)
    srcs = bench.pick_sources(deg, 16, seed=2022 + rank)
    assert (deg[srcs] > 0).all()
    local_time = 1.0 + rank          # rank 1 is the slowest
    local_work = 100 * (rank + 1)
    d.barrier()
    t = d.max(local_time)
    w = d.sum(local_work)
    q.put((rank, t, w, srcs.tolist()))
    dist.destroy_process_group()


def test_two_rank_aggregation_gloo():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    res.sort()
    for rank, t, w, _ in res:
        assert t == 2.0          # max over ranks
        assert w == 300          # sum over ranks
    assert res[0][3] != res[1][3]  # replicas traverse different sources
