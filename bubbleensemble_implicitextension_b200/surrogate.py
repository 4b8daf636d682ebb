"""Learned screening of amplitude x frequency sweeps.

A small MLP (6 -> 256 x 4 GELU -> 2, the library's own CUDA kernels, BF16
with FP32 master weights, Adam) maps a system's drive and bubble-size
statistics to its collapse outputs:

    inputs  (pressure amplitude [bar], log10 frequency [kHz],
             mean, std, min, max of the equilibrium radii [um])
    outputs (log10 collapse strength, max R/R_E)

where, over the recorded periods, collapse strength is the largest
Rmax_k / Rmin_k of any bubble and max R/R_E the largest recorded radius
maximum.  The training data come from the solver itself (:func:`generate_runs`).
:func:`screen_sweep` predicts a whole sweep map, flags the points where the
prediction changes steeply between grid neighbours plus a random audit
sample, integrates only those with the solver, and serves the rest from the
network; the audit measures the error of what the network served.
:func:`screen_sweep_lattice` is the multi-fidelity form used by the sweep
benchmark: the solver integrates a coarse lattice of the grid, the network's
map is corrected by the bilinearly interpolated lattice residuals, and every
lattice cell whose corners disagree, or where the corrected network departs
from plain interpolation of the corners, is integrated in full.
"""
from __future__ import annotations

import ctypes
import dataclasses
import time
from typing import Callable, Optional

import numpy as np

from . import solver as S
from . import workloads as W

N_IN, N_OUT = 6, 2


def _fp(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_float))


class MLP:
    """The surrogate network on one GPU (bes_mlp_* of include/bes.h).

    Inputs and outputs of forward/backward are torch CUDA float32 tensors
    ([batch, 6] and [batch, 2])."""

    def __init__(self, n_in=N_IN, width=256, depth=4, n_out=N_OUT, max_batch=4096, seed=0, device=0):
        self._lib = S.load_library()
        cfg = S.MlpConfig(device, n_in, width, depth, n_out, max_batch, seed)
        h = ctypes.c_void_p()
        st = self._lib.bes_mlp_create(ctypes.byref(cfg), ctypes.byref(h))
        if st != 0:
            raise S.BesError(st, "bes_mlp_create failed")
        self._h = h
        self.n_in, self.width, self.depth, self.n_out, self.max_batch = n_in, width, depth, n_out, max_batch
        n = ctypes.c_int64()
        self._ok(self._lib.bes_mlp_parameter_count(self._h, ctypes.byref(n)))
        self.n_params = n.value
        self.sizes = [(n_in if l == 0 else width, n_out if l == depth else width) for l in range(depth + 1)]
        self.norm = (np.zeros(n_in, np.float32), np.ones(n_in, np.float32), np.zeros(n_out, np.float32),
                     np.ones(n_out, np.float32))

    def _ok(self, st):
        if st != 0:
            raise S.BesError(st, self._lib.bes_mlp_last_error(self._h).decode())

    def close(self):
        if getattr(self, "_h", None):
            self._lib.bes_mlp_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_normalization(self, in_mean, in_std, out_mean, out_std):
        arrs = [np.ascontiguousarray(a, np.float32) for a in (in_mean, in_std, out_mean, out_std)]
        self.norm = tuple(arrs)
        self._ok(self._lib.bes_mlp_set_normalization(self._h, *[_fp(a) for a in arrs]))

    def parameters(self) -> np.ndarray:
        out = np.empty(self.n_params, np.float32)
        self._ok(self._lib.bes_mlp_get_parameters(self._h, _fp(out), out.size))
        return out

    def set_parameters(self, p: np.ndarray):
        p = np.ascontiguousarray(p, np.float32)
        self._ok(self._lib.bes_mlp_set_parameters(self._h, _fp(p), p.size))

    def gradients(self) -> np.ndarray:
        out = np.empty(self.n_params, np.float32)
        self._ok(self._lib.bes_mlp_get_gradients(self._h, _fp(out), out.size))
        return out

    def forward(self, x):
        import torch
        y = torch.empty((x.shape[0], self.n_out), dtype=torch.float32, device=x.device)
        stream = torch.cuda.current_stream(x.device).cuda_stream
        for b0 in range(0, x.shape[0], self.max_batch):
            xb = x[b0:b0 + self.max_batch].contiguous()
            yb = y[b0:b0 + self.max_batch]
            self._ok(self._lib.bes_mlp_forward(self._h, xb.data_ptr(), xb.shape[0], yb.data_ptr(),
                                               ctypes.c_void_p(stream)))
        return y

    def backward(self, x, t) -> float:
        import torch
        loss = ctypes.c_float()
        stream = torch.cuda.current_stream(x.device).cuda_stream
        self._ok(self._lib.bes_mlp_backward(self._h, x.contiguous().data_ptr(), t.contiguous().data_ptr(),
                                            x.shape[0], ctypes.byref(loss), ctypes.c_void_p(stream)))
        return loss.value

    def adam_step(self, lr: float):
        import torch
        self._ok(self._lib.bes_mlp_adam_step(self._h, ctypes.c_float(lr),
                                             ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)))

    def fit(self, X: np.ndarray, Y: np.ndarray, steps: int = 3000, batch: int = 512, lr: float = 2e-3,
            seed: int = 0, log_every: int = 0) -> list:
        """Adam on minibatches with a cosine learning-rate decay; standardises with the data's statistics."""
        import torch
        self.set_normalization(X.mean(0), X.std(0) + 1e-6, Y.mean(0), Y.std(0) + 1e-6)
        dev = torch.device("cuda", torch.cuda.current_device())
        Xt = torch.as_tensor(X, dtype=torch.float32, device=dev)
        Yt = torch.as_tensor(Y, dtype=torch.float32, device=dev)
        rng = np.random.default_rng(seed)
        hist = []
        for it in range(steps):
            idx = torch.as_tensor(rng.integers(0, len(X), min(batch, len(X))), device=dev)
            loss = self.backward(Xt[idx], Yt[idx])
            self.adam_step(lr * 0.5 * (1.0 + np.cos(np.pi * it / steps)))
            if log_every and it % log_every == 0:
                hist.append((it, loss))
        return hist

    def predict(self, X: np.ndarray) -> np.ndarray:
        import torch
        dev = torch.device("cuda", torch.cuda.current_device())
        return self.forward(torch.as_tensor(X, dtype=torch.float32, device=dev)).cpu().numpy()


# ---- solver-generated data --------------------------------------------------

def features(pa_bar, f_khz, radii_um) -> np.ndarray:
    """[amplitude, log10 frequency, mean, std, min, max of the radii] per system."""
    r = np.asarray(radii_um, np.float64)
    if r.ndim == 1:
        r = np.broadcast_to(r, (len(np.atleast_1d(pa_bar)), r.size))
    return np.stack([np.asarray(pa_bar, np.float64), np.log10(np.asarray(f_khz, np.float64)), r.mean(1), r.std(1),
                     r.min(1), r.max(1)], axis=1)


def labels(uacc: np.ndarray, iuacc: np.ndarray, units: np.ndarray) -> np.ndarray:
    """[log10 max collapse strength, max recorded R/R_E] per system (1 and 0 when nothing was recorded)."""
    rmax, rmin, strength, count = W.collapse_records(uacc, iuacc, units)
    off = np.concatenate([[0], np.cumsum(units)])
    n = len(units)
    out = np.zeros((n, 2))
    nrec = np.clip(count, 0, W.NCOLL)
    slot = np.arange(W.NCOLL)[:, None]
    valid = slot < nrec[None, :]
    s_masked = np.where(valid, strength, 0.0).max(0)
    r_masked = np.where(valid, rmax, 0.0).max(0)
    for s in range(n):
        a, b = off[s], off[s + 1]
        out[s, 0] = np.log10(max(s_masked[a:b].max(), 1.0))
        out[s, 1] = r_masked[a:b].max()
    return out


def line_ensemble(pa_bar, f_khz, radii_per_system, spacing_um=150.0, n_periods=8, reset_at=4,
                  rtol=1e-10) -> W.Ensemble:
    """N-bubble line systems (one radius draw per system) at the given drives."""
    pa = np.asarray(pa_bar, np.float64)
    fr = np.asarray(f_khz, np.float64)
    R = np.asarray(radii_per_system, np.float64)
    ns, n = R.shape
    pos = spacing_um * np.arange(n)
    coup = np.concatenate([W.coupling_from_geometry(pos, R[s]).T.reshape(-1) for s in range(ns)])
    up = W.km_unit_parameters(pa[:, None], fr[:, None], 0.0, 0.0, 0.0, R).reshape(W.NUP, ns * n)
    st = np.zeros((2, ns * n))
    st[0] = 1.0
    return W.Ensemble(units=np.full(ns, n, np.int32), upar=up, state=st, coupling=coup,
                      matrix_of_system=np.arange(ns, dtype=np.int32), rtol=np.full((2, ns), rtol),
                      atol=np.full((2, ns), rtol), n_periods=n_periods, reset_at=reset_at, name="line")


def solve_ensemble(ens: W.Ensemble, max_steps: int = 50_000, device: int = 0):
    """Integrate with the library; returns (labels, status, seconds of the solve)."""
    ens.max_steps_per_period = max_steps
    ps = ens.make_solver(device=device)
    try:
        V = S.ListOfVariables
        ps.SynchroniseFromHostToDevice(V.All)
        ps.InsertSynchronisationPoint()
        ps.SynchroniseSolver()
        t0 = time.perf_counter()
        ps.solve_periods(ens.n_periods, ens.reset_at)
        ps.InsertSynchronisationPoint()
        ps.SynchroniseSolver()
        dt = time.perf_counter() - t0
        ps.SynchroniseFromDeviceToHost(V.All)
        ps.InsertSynchronisationPoint()
        ps.SynchroniseSolver()
        uacc = ps.get_array(V.UnitAccessories).reshape(W.NUA, -1)
        iuacc = ps.get_array(V.IntegerUnitAccessories).reshape(1, -1)
        status = ps.counters()["status"]
    finally:
        ps.close()
    return labels(uacc, iuacc, ens.units), status, dt


def generate_runs(n_runs: int, seed: int = 7, n_units: int = 32, n_periods: int = 8, reset_at: int = 4,
                  pa_range=(0.5, 2.0), f_range=(20.0, 200.0), radius_range=(2.0, 8.0), device: int = 0):
    """Training data from the solver: random amplitude (uniform), frequency
    (log-uniform) and radii (uniform, one draw per run) on the 150 um line."""
    rng = np.random.default_rng(seed)
    pa = rng.uniform(*pa_range, n_runs)
    fr = 10 ** rng.uniform(np.log10(f_range[0]), np.log10(f_range[1]), n_runs)
    R = rng.uniform(*radius_range, (n_runs, n_units))
    ens = line_ensemble(pa, fr, R, n_periods=n_periods, reset_at=reset_at)
    Y, status, dt = solve_ensemble(ens, device=device)
    return features(pa, fr, R), Y, status, dt


@dataclasses.dataclass
class ScreenResult:
    map: np.ndarray            # served values [n_pa, n_f, 2]
    integrated: np.ndarray     # bool [n_pa, n_f]: integrated by the solver
    audited: np.ndarray        # bool [n_pa, n_f]: random audit points (also integrated)
    audit_max_rel_error: float # network error on the audit sample, log10 strength
    seconds: float


def screen_sweep(mlp: MLP, pa: np.ndarray, f_khz: np.ndarray, radii_um: np.ndarray,
                 solve: Callable[[np.ndarray, np.ndarray], np.ndarray], grad_quantile: float = 0.75,
                 audit_fraction: float = 0.02, seed: int = 0) -> ScreenResult:
    """Predict the whole grid, integrate the steep and audit points, serve the rest.

    `solve(pa_points, f_points)` must return the solver's outputs [n, 2] for the
    listed points.  A point is steep when the predicted log10 strength differs
    from a grid neighbour by more than the `grad_quantile` quantile of those
    differences over the map."""
    t0 = time.perf_counter()
    PA, FR = np.meshgrid(pa, f_khz, indexing="ij")
    X = features(PA.ravel(), FR.ravel(), radii_um)
    pred = mlp.predict(X).reshape(len(pa), len(f_khz), 2).astype(np.float64)
    m = pred[..., 0]
    jump = np.zeros_like(m)
    jump[1:, :] = np.maximum(jump[1:, :], np.abs(m[1:, :] - m[:-1, :]))
    jump[:-1, :] = np.maximum(jump[:-1, :], np.abs(m[1:, :] - m[:-1, :]))
    jump[:, 1:] = np.maximum(jump[:, 1:], np.abs(m[:, 1:] - m[:, :-1]))
    jump[:, :-1] = np.maximum(jump[:, :-1], np.abs(m[:, 1:] - m[:, :-1]))
    steep = jump > np.quantile(jump, grad_quantile)
    rng = np.random.default_rng(seed)
    audit = rng.random(m.shape) < audit_fraction
    todo = steep | audit
    out = pred.copy()
    vals = solve(PA[todo], FR[todo])
    out[todo] = vals
    a_idx = audit & ~steep
    err = 0.0
    if a_idx.any():
        sol = out[a_idx][:, 0]
        err = float(np.max(np.abs(pred[a_idx][:, 0] - sol) / np.maximum(np.abs(sol), 1e-3)))
    return ScreenResult(map=out, integrated=todo, audited=audit, audit_max_rel_error=err,
                        seconds=time.perf_counter() - t0)


@dataclasses.dataclass
class LatticeScreenResult:
    map: np.ndarray            # served values [n_pa, n_f, 2]
    integrated: np.ndarray     # bool [n_pa, n_f]: the solver's values (lattice, flagged cells, audit)
    lattice: np.ndarray        # bool [n_pa, n_f]: lattice points
    audited: np.ndarray        # bool [n_pa, n_f]: audit points outside flagged cells
    audit_max_rel_error: float # corrected-network error on the audit points, collapse strength
    solve_seconds: float       # time inside the solver (all passes)
    seconds: float             # whole screened sweep (without the verification pass)
    served_map: Optional[np.ndarray] = None     # with verify: what the screener would have served [n_pa, n_f, 2]
    verify_seconds: float = 0.0                 # with verify: the pass that integrates every served point
    served_rel_error: Optional[np.ndarray] = None  # with verify: |served - solver| / solver per point, strength


def _lattice_axis(n: int, stride: int):
    """Lattice indices of one grid axis (every stride-th point and the last one)
    and, per grid point, its cell index and bilinear weight."""
    idx = np.unique(np.r_[np.arange(0, n, stride), n - 1])
    cell = np.clip(np.searchsorted(idx, np.arange(n), side="right") - 1, 0, len(idx) - 2)
    t = (np.arange(n) - idx[cell]) / (idx[cell + 1] - idx[cell])
    return idx, cell, t


def screen_sweep_lattice(mlp: Optional["MLP"], pa: np.ndarray, f_khz: np.ndarray, radii_um: np.ndarray,
                         solve: Callable[[np.ndarray, np.ndarray], np.ndarray], stride: int = 4,
                         cell_spread: float = 0.05, cell_disagreement: float = 0.02,
                         audit_fraction: float = 0.02, seed: int = 0, verify: bool = False) -> LatticeScreenResult:
    """Multi-fidelity sweep: solver lattice + network corrected by the lattice residuals.

    `solve(pa_points, f_points)` returns the solver's outputs [n, 2] (log10
    collapse strength, max R/R_E).  A lattice cell is integrated in full when
    its corner strengths spread by more than `cell_spread` (relative), or when
    the corrected network strength differs from the bilinear interpolation of
    the corner solutions by more than `cell_disagreement` (relative) anywhere
    inside it; a random `audit_fraction` of the other points is integrated too
    and measures the error of what is served.

    mlp=None is the same screener without the network: the served values are
    the bilinear interpolation of the lattice solutions and only the corner
    spread flags cells (what the network adds is the difference between the
    two runs).  verify=True integrates every served point as well, after the
    screened map is complete: the map returned is then the solver's everywhere,
    served_map and served_rel_error record what the screener had served and
    how far it was off, and verify_seconds the cost of that pass."""
    t0 = time.perf_counter()
    n_pa, n_f = len(pa), len(f_khz)
    PA, FR = np.meshgrid(pa, f_khz, indexing="ij")
    ia, ca, ta = _lattice_axis(n_pa, stride)
    ib, cb, tb = _lattice_axis(n_f, stride)
    lat = np.zeros((n_pa, n_f), bool)
    lat[np.ix_(ia, ib)] = True
    solve_s = 0.0
    t1 = time.perf_counter()
    sol = np.zeros((n_pa, n_f, 2))
    sol[lat] = solve(PA[lat], FR[lat])
    solve_s += time.perf_counter() - t1
    if mlp is not None:
        pred = mlp.predict(features(PA.ravel(), FR.ravel(), radii_um)).reshape(n_pa, n_f, 2).astype(np.float64)
    else:
        pred = np.zeros((n_pa, n_f, 2))   # no network: the residuals are the lattice solutions themselves
    res = np.where(lat[..., None], sol - pred, 0.0)
    # bilinear interpolation inside each cell: corners (a, b), (a+1, b), (a, b+1), (a+1, b+1)
    A0, A1 = ia[ca][:, None], ia[ca + 1][:, None]
    B0, B1 = ib[cb][None, :], ib[cb + 1][None, :]
    wa, wb = ta[:, None, None], tb[None, :, None]

    def bil(v):
        return ((1 - wa) * (1 - wb) * v[A0, B0] + wa * (1 - wb) * v[A1, B0] + (1 - wa) * wb * v[A0, B1]
                + wa * wb * v[A1, B1])

    corr = pred + bil(res)
    interp = bil(sol)
    # per cell: corner spread of the strength and the largest corrected-vs-interpolated departure
    nca, ncb = len(ia) - 1, len(ib) - 1
    cs = sol[..., 0]
    corners = np.stack([cs[np.ix_(ia[:-1], ib[:-1])], cs[np.ix_(ia[1:], ib[:-1])], cs[np.ix_(ia[:-1], ib[1:])],
                        cs[np.ix_(ia[1:], ib[1:])]])
    spread = 10.0 ** (corners.max(0) - corners.min(0)) - 1.0
    dep = np.abs(10.0 ** (corr[..., 0] - interp[..., 0]) - 1.0)
    dep_cell = np.zeros((nca, ncb))
    np.maximum.at(dep_cell, (np.broadcast_to(ca[:, None], dep.shape), np.broadcast_to(cb[None, :], dep.shape)), dep)
    bad = (spread > cell_spread) | (dep_cell > cell_disagreement)
    flag = np.zeros((n_pa, n_f), bool)
    for a, b in np.argwhere(bad):
        flag[ia[a]:ia[a + 1] + 1, ib[b]:ib[b + 1] + 1] = True
    rng = np.random.default_rng(seed)
    audit = (rng.random((n_pa, n_f)) < audit_fraction) & ~flag & ~lat
    todo = (flag | audit) & ~lat
    t1 = time.perf_counter()
    if todo.any():
        sol[todo] = solve(PA[todo], FR[todo])
    solve_s += time.perf_counter() - t1
    integrated = lat | todo
    out = np.where(integrated[..., None], sol, corr)
    err = 0.0
    if audit.any():
        s_true = 10.0 ** sol[audit][:, 0]
        err = float(np.max(np.abs(10.0 ** corr[audit][:, 0] - s_true) / s_true))
    seconds = time.perf_counter() - t0
    result = LatticeScreenResult(map=out, integrated=integrated, lattice=lat, audited=audit,
                                 audit_max_rel_error=err, solve_seconds=solve_s, seconds=seconds)
    if verify:
        served = ~integrated
        t1 = time.perf_counter()
        checked = sol.copy()
        if served.any():
            checked[served] = solve(PA[served], FR[served])
        result.verify_seconds = time.perf_counter() - t1
        s_true = 10.0 ** checked[..., 0]
        result.served_rel_error = np.where(served, np.abs(10.0 ** out[..., 0] - s_true) / s_true, 0.0)
        result.served_map = out
        result.map = checked
    return result
