"""Sharding an ensemble or a sweep over GPUs, one process per GPU.

Systems are independent: the integration has no exchange step, and the
reference ran one separate job per device (JobGenerationAndSubmission.sh:
4-31).  A shard is therefore a contiguous range of systems, chosen so that
the ranks' costs balance, and the only collective is the gather of the result
records on rank 0 after the solve.

The cost of a system is what its integration takes, which the unit count
alone does not predict (two systems of the same size can differ tenfold in
their number of steps).  ``pilot_costs`` measures it: every rank integrates an
even share of the systems once (a pilot period, or a shorter one), the
attempted steps times the per-step work of the system's size are gathered,
and ``cost_bounds`` cuts the ensemble at equal shares of the total.

The functions take ``torch.distributed`` as the transport (NCCL on the GPUs,
gloo on the CPU); with ``world == 1`` they need no process group.
"""
from __future__ import annotations

from typing import Callable, Dict, Optional

import numpy as np

from . import workloads as W


def step_work(units: np.ndarray) -> np.ndarray:
    """Relative work of one attempted step of a system of N units: six
    right-hand sides whose BiCG products cost ~N^2, plus per-unit work ~N."""
    n = np.asarray(units, np.float64)
    return n * n + 16.0 * n


def cost_bounds(cost: np.ndarray, world: int) -> np.ndarray:
    """Contiguous partition of systems into `world` shards of nearly equal total
    cost: rank r takes systems [bounds[r], bounds[r + 1]).  A cut falls after
    the system at which the running cost first reaches r / world of the total,
    so no shard is empty while systems remain."""
    c = np.asarray(cost, np.float64)
    n = len(c)
    cum = np.cumsum(c)
    total = cum[-1] if n else 0.0
    cuts = [0]
    for r in range(1, world):
        k = int(np.searchsorted(cum, total * r / world, side="left")) + 1
        cuts.append(min(max(k, cuts[-1]), n))
    cuts.append(n)
    return np.asarray(cuts, np.int64)


def even_bounds(n: int, world: int) -> np.ndarray:
    """Contiguous partition of n systems into shares of equal count."""
    return np.asarray([(n * r) // world for r in range(world + 1)], np.int64)


def _all_gather_object(obj, world: int):
    if world == 1:
        return [obj]
    import torch.distributed as dist
    out = [None] * world
    dist.all_gather_object(out, obj)
    return out


def pilot_costs(ens: W.Ensemble, rank: int, world: int,
                solve: Callable[[W.Ensemble], Dict[str, np.ndarray]]) -> np.ndarray:
    """Measured per-system cost, the same array on every rank.

    Rank r integrates systems [even_bounds[r], even_bounds[r + 1]) with
    `solve` (which returns per-system counters "n_accepted" and "n_rejected");
    the cost is the attempted steps times ``step_work`` of the system's size."""
    b = even_bounds(ens.n_systems, world)
    mine = list(range(int(b[rank]), int(b[rank + 1])))
    if mine:
        out = solve(ens.subset(mine))
        att = np.asarray(out["n_accepted"], np.float64) + np.asarray(out["n_rejected"], np.float64)
    else:
        att = np.zeros(0)
    parts = _all_gather_object(att, world)
    attempted = np.concatenate([np.asarray(p, np.float64) for p in parts])
    return np.maximum(attempted, 1.0) * step_work(ens.units)


def shard(ens: W.Ensemble, bounds: np.ndarray, rank: int) -> W.Ensemble:
    """Rank `rank`'s contiguous share."""
    return ens.subset(list(range(int(bounds[rank]), int(bounds[rank + 1]))))


# result arrays and the axis they run along: per unit (columns of [k][total_units]) or per system
UNIT_KEYS = ("state", "uacc", "iuacc")
SYSTEM_KEYS = ("n_accepted", "n_rejected", "n_bicg_iter", "n_rhs", "status", "actual_time")


def gather_results(local: Dict[str, np.ndarray], rank: int, world: int) -> Optional[Dict[str, np.ndarray]]:
    """The shards' result records concatenated in system order on rank 0
    (None on the other ranks).  Unit-scope arrays [k][units of the shard] are
    joined along the unit axis, system-scope arrays along the system axis."""
    rec = {k: np.asarray(local[k]) for k in UNIT_KEYS + SYSTEM_KEYS if k in local}
    if world == 1:
        return rec
    import torch.distributed as dist
    parts = [None] * world if rank == 0 else None
    dist.gather_object(rec, parts, dst=0)
    if rank != 0:
        return None
    out = {}
    for k in rec:
        axis = -1 if k in UNIT_KEYS else 0
        out[k] = np.concatenate([p[k] for p in parts], axis=axis)
    return out


def sharded_points_solve(solve: Callable[[np.ndarray, np.ndarray], np.ndarray], rank: int, world: int,
                         cost: Optional[Callable[[np.ndarray, np.ndarray], np.ndarray]] = None):
    """A sweep's solve callback split over the ranks: the requested points are cut
    into contiguous shares (of equal count, or of equal estimated cost when
    `cost(pa, f)` gives one per point), each rank integrates its share with
    `solve`, and the outputs are all-gathered so that every rank returns the
    full [n, k] array.  Every rank must call it with the same points in the
    same order (the sweep screener is deterministic, so it does)."""
    if world == 1:
        return solve

    def run(pa_pts: np.ndarray, f_pts: np.ndarray) -> np.ndarray:
        n = len(pa_pts)
        b = cost_bounds(cost(pa_pts, f_pts), world) if cost is not None else even_bounds(n, world)
        lo, hi = int(b[rank]), int(b[rank + 1])
        mine = solve(pa_pts[lo:hi], f_pts[lo:hi]) if hi > lo else None
        parts = _all_gather_object(None if mine is None else np.asarray(mine), world)
        return np.concatenate([p for p in parts if p is not None], axis=0)

    return run
