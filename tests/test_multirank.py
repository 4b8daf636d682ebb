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


def _shard_worker(rank, world, port, out):
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank), MASTER_ADDR="127.0.0.1",
                      MASTER_PORT=str(port))
    import datetime

    import torch.distributed as dist

    from bubbleensemble_implicitextension_b200 import sharding as SH
    from bubbleensemble_implicitextension_b200 import workloads as W
    from oracle import oracle as O

    dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=120))
    ens = W.c1_ensemble().subset(list(range(0, 256, 21)))
    ens.max_steps_per_period = 50_000
    solve = lambda e: O.run(e, n_periods=1, reset_at=-1, threads=1)  # noqa: E731  (the CPU stand-in of a GPU)
    cost = SH.pilot_costs(ens, rank, world, solve)
    bounds = SH.cost_bounds(cost, world)
    part = SH.shard(ens, bounds, rank)
    res = SH.gather_results(solve(part), rank, world)
    out[rank] = (bounds.tolist(), cost.tolist(), res)
    dist.destroy_process_group()


@pytest.mark.timeout(600)
def test_sharded_solve_gathers_the_single_rank_result():
    """Two gloo ranks: a pilot measures per-system cost, the ensemble is cut into
    two contiguous cost-balanced shards, each rank integrates its shard (the
    oracle stands in for the GPU), and the records gathered on rank 0 equal the
    single-rank run bit for bit."""
    from bubbleensemble_implicitextension_b200 import sharding as SH
    from bubbleensemble_implicitextension_b200 import workloads as W
    from oracle import oracle as O

    ctx = mp.get_context("spawn")
    with ctx.Manager() as mgr:
        out = mgr.dict()
        port = _free_port()
        procs = [ctx.Process(target=_shard_worker, args=(r, 2, port, out)) for r in range(2)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(540)
            assert p.exitcode == 0
        res = dict(out)
    bounds, cost, gathered = res[0]
    assert res[1][2] is None and res[1][0] == bounds
    ens = W.c1_ensemble().subset(list(range(0, 256, 21)))
    ens.max_steps_per_period = 50_000
    whole = O.run(ens, n_periods=1, reset_at=-1)
    for k in SH.UNIT_KEYS + SH.SYSTEM_KEYS:
        np.testing.assert_array_equal(gathered[k], np.asarray(whole[k]), err_msg=k)
    # the cut balances the measured cost to within the cost of one system
    c = np.asarray(cost)
    shares = [c[bounds[r]:bounds[r + 1]].sum() for r in range(2)]
    assert 0 < bounds[1] < ens.n_systems
    assert max(shares) - min(shares) <= c.max()


def test_cost_bounds_properties():
    from bubbleensemble_implicitextension_b200 import sharding as SH
    rng = np.random.default_rng(0)
    for world in (1, 2, 3, 8):
        for n in (0, 1, 5, 100):
            c = rng.uniform(0.1, 10.0, n)
            b = SH.cost_bounds(c, world)
            assert b[0] == 0 and b[-1] == n and len(b) == world + 1
            assert (np.diff(b) >= 0).all()
            if n >= world:
                shares = [c[b[r]:b[r + 1]].sum() for r in range(world)]
                assert max(shares) - c.sum() / world <= c.max() + 1e-9


def _sweep_worker(rank, world, port, out):
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank), MASTER_ADDR="127.0.0.1",
                      MASTER_PORT=str(port))
    import datetime

    import torch.distributed as dist

    from bubbleensemble_implicitextension_b200 import sharding as SH
    from bubbleensemble_implicitextension_b200 import surrogate as SG
    from tests.test_sweep_screen import _Net, _grid, _map

    dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=120))
    calls = []

    def solve_local(pp, ff):
        calls.append(len(pp))
        return _map(pp, ff, True)

    pa, f = _grid()
    solve = SH.sharded_points_solve(solve_local, rank, world)
    res = SG.screen_sweep_lattice(_Net(), pa, f, np.full(32, 5.0), solve, stride=4, cell_spread=0.5,
                                  cell_disagreement=0.05, audit_fraction=0.05, seed=2)
    out[rank] = (res.map, res.integrated, sum(calls))
    dist.destroy_process_group()


@pytest.mark.timeout(300)
def test_sharded_sweep_screen_equals_single_rank():
    """The sweep screener with its solves split over two gloo ranks: both ranks end
    with the single-rank map, and the points were shared between them."""
    from bubbleensemble_implicitextension_b200 import surrogate as SG
    from tests.test_sweep_screen import _Net, _grid, _map

    ctx = mp.get_context("spawn")
    with ctx.Manager() as mgr:
        out = mgr.dict()
        port = _free_port()
        procs = [ctx.Process(target=_sweep_worker, args=(r, 2, port, out)) for r in range(2)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(240)
            assert p.exitcode == 0
        res = dict(out)
    pa, f = _grid()
    single = SG.screen_sweep_lattice(_Net(), pa, f, np.full(32, 5.0), lambda pp, ff: _map(pp, ff, True), stride=4,
                                     cell_spread=0.5, cell_disagreement=0.05, audit_fraction=0.05, seed=2)
    for r in range(2):
        np.testing.assert_array_equal(res[r][0], single.map)
        np.testing.assert_array_equal(res[r][1], single.integrated)
    assert res[0][2] + res[1][2] == int(single.integrated.sum())   # each point integrated once, on one rank
    assert res[0][2] > 0 and res[1][2] > 0
