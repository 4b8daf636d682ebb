"""Shared helpers: run an ensemble through the library (GPU) or the oracle (CPU)."""
import numpy as np

from bubbleensemble_implicitextension_b200 import solver as S
from bubbleensemble_implicitextension_b200 import workloads as W

V = S.ListOfVariables
O = S.ListOfSolverOptions


def run_gpu(ens, n_periods=None, reset_at=None, algorithm=S.Algorithms.RKCK45, ndo=0, do_min_dt=0.0,
            do_save_frequency=1, per_period_solve=False, warps_per_block=0, bicg_max_iter=19, use_graph=True,
            repeat=1, shared_matrices=False, warps_per_system=0, autotune=False, bicg_recurrence=0):
    n_periods = ens.n_periods if n_periods is None else n_periods
    reset_at = ens.reset_at if reset_at is None else reset_at
    ps = ens.make_solver(algorithm=algorithm, n_dense_output=ndo)
    try:
        if ndo:
            ps.SolverOption(O.DenseOutputMinimumTimeStep, do_min_dt)
            ps.SolverOption(O.DenseOutputSaveFrequency, do_save_frequency)
        if warps_per_block:
            ps.SolverOption(O.WarpsPerBlock, warps_per_block)
        if bicg_max_iter != 19:
            ps.SolverOption(O.BiCGMaxIterations, bicg_max_iter)
        if not use_graph:
            ps.SolverOption(O.UseCudaGraph, 0)
        if shared_matrices:
            ps.SolverOption(O.SharedCouplingMatrices, 1)
        if warps_per_system:
            ps.SolverOption(O.WarpsPerSystem, warps_per_system)
        if bicg_recurrence:
            ps.SolverOption(O.BiCGRecurrence, bicg_recurrence)
        for _ in range(repeat - 1):       # earlier solves whose results are discarded (graph capture, replays)
            ps.SynchroniseFromHostToDevice(V.All)
            ps.solve_periods(n_periods, reset_at)
            ps.reset_counters()
        ps.SynchroniseFromHostToDevice(V.All)
        if autotune:
            out_tune = ps.autotune(n_periods=1, step_cap=300)
            assert out_tune["candidates"] >= 1
        if per_period_solve:
            for p in range(n_periods):
                if p == reset_at:
                    ps.set_array(V.UnitAccessories, np.zeros((64, ens.total_units)))
                    ps.set_array(V.IntegerUnitAccessories, np.full(ens.total_units, -1, np.int32))
                    ps.SynchroniseFromHostToDevice(V.UnitAccessories)
                    ps.SynchroniseFromHostToDevice(V.IntegerUnitAccessories)
                ps.Solve()
                ps.InsertSynchronisationPoint()
                ps.SynchroniseSolver()
        else:
            ps.solve_periods(n_periods, reset_at)
        ps.SynchroniseFromDeviceToHost(V.All)
        ps.InsertSynchronisationPoint()
        ps.SynchroniseSolver()
        out = {
            "state": ps.get_array(V.ActualState).reshape(2, -1),
            "uacc": ps.get_array(V.UnitAccessories).reshape(64, -1),
            "iuacc": ps.get_array(V.IntegerUnitAccessories).reshape(1, -1),
            "actual_time": ps.get_array(V.ActualTime),
        }
        c = ps.counters()
        out.update({"n_accepted": c["accepted"].astype(np.int64), "n_rejected": c["rejected"].astype(np.int64),
                    "n_bicg_iter": c["bicg"].astype(np.int64), "n_rhs": c["rhs"].astype(np.int64),
                    "status": c["status"]})
        if ndo:
            out["dense_index"] = ps.get_array(V.DenseIndex)
            out["dense_time"] = ps.get_array(V.DenseTime).reshape(ndo, -1)
            out["dense_state"] = ps.get_array(V.DenseState).reshape(ndo, 2, -1)
        return out
    finally:
        ps.close()


def max_rel(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    d = np.abs(a - b) / np.maximum(np.abs(b), 1e-300)
    d[(a == b)] = 0.0
    return float(np.nanmax(d)) if d.size else 0.0


def assert_bitwise(got, want, keys):
    for k in keys:
        g, w = np.asarray(got[k]), np.asarray(want[k])
        assert g.shape == w.shape, (k, g.shape, w.shape)
        if g.dtype.kind == "f":
            same = (g.view(np.int64) == w.view(np.int64)) | (np.isnan(g) & np.isnan(w))
        else:
            same = g == w
        if not same.all():
            idx = np.argwhere(~same)[:5]
            raise AssertionError(f"{k}: {int((~same).sum())} of {same.size} entries differ, first at {idx.tolist()}, "
                                 f"max rel {max_rel(g, w):.3e}")


def ragged_ensemble(sizes, seed=11, n_periods=1, reset_at=-1, rtol=1e-10, pa=(0.6, 1.4), f=(60.0, 200.0)):
    """Small uneven ensemble: one random 3-D cloud per system."""
    rng = np.random.default_rng(seed)
    ups, coups, states = [], [], []
    for n in sizes:
        pts = rng.uniform(0.0, 80.0 * n ** (1 / 3) + 100.0, (n, 3))
        r = rng.uniform(2.0, 8.0, n)
        up = W.km_unit_parameters(rng.uniform(*pa), rng.uniform(*f), 0.0, 0.0, 0.0, r)
        ups.append(up)
        coups.append(W.coupling_from_geometry(pts, r).T.reshape(-1))
        st = np.zeros((2, n))
        st[0] = 1.0
        states.append(st)
    ns = len(sizes)
    return W.Ensemble(units=np.asarray(sizes, np.int32), upar=np.concatenate(ups, 1), state=np.concatenate(states, 1),
                      coupling=np.concatenate(coups), matrix_of_system=np.arange(ns, dtype=np.int32),
                      rtol=np.full((2, ns), rtol), atol=np.full((2, ns), rtol), n_periods=n_periods,
                      reset_at=reset_at, name="ragged")
