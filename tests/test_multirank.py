"""The multi-GPU host path on CPU: two gloo ranks (127.0.0.1) run the bench's
timing reduction and barrier, and shard an uneven ensemble contiguously by
cost; every system lands on exactly one rank and the shares are balanced."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, out):
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank), MASTER_ADDR="127.0.0.1",
                      MASTER_PORT=str(port))
    import torch
    import torch.distributed as dist

    import bench
    from bubbleensemble_implicitextension_b200 import workloads as W

    r, w, _ = bench.dist_init(world)
    assert (r, w) == (rank, world)
    bench.barrier(w)
    t = bench.allreduce_max(10.0 + rank, w)              # the slowest rank's time
    ens = W.c2_ensemble(n_systems=300, seed=5)
    part = W.shard(ens, rank, world)
    b = W.shard_bounds(ens.units, world)
    mine = torch.tensor([b[rank], b[rank + 1], part.n_systems, int((part.units.astype(np.int64) ** 2).sum())],
                        dtype=torch.int64)
    gathered = [torch.zeros(4, dtype=torch.int64) for _ in range(w)]
    dist.all_gather(gathered, mine)
    out[rank] = (t, [g.tolist() for g in gathered], ens.n_systems)
    dist.destroy_process_group()


@pytest.mark.timeout(300)
def test_two_gloo_ranks_reduce_and_shard():
    ctx = mp.get_context("spawn")
    with ctx.Manager() as mgr:
        out = mgr.dict()
        port = _free_port()
        procs = [ctx.Process(target=_worker, args=(r, 2, port, out)) for r in range(2)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(240)
            assert p.exitcode == 0
        res = dict(out)
    for r in range(2):
        t, shards, n = res[r]
        assert t == 11.0
        assert shards[0][0] == 0 and shards[0][1] == shards[1][0] and shards[1][1] == n
        assert shards[0][2] + shards[1][2] == n
        c0, c1 = shards[0][3], shards[1][3]
        assert abs(c0 - c1) <= 0.05 * (c0 + c1)            # cost-balanced within 5 %
