"""TEST INFRASTRUCTURE: ctypes binding of the CPU oracle ``liboracle.so``.

Only the tests, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` use this module; the product never imports it.  The oracle is a
plain C++ FP64 restatement of the reference's per-block solver (see
bes_oracle.h for the reference file:line of each part).
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB = HERE / "liboracle.so"

_i32p = ctypes.POINTER(ctypes.c_int32)
_i64p = ctypes.POINTER(ctypes.c_int64)
_dp = ctypes.POINTER(ctypes.c_double)


class Problem(ctypes.Structure):
    _fields_ = [
        ("n_systems", ctypes.c_int32), ("active_systems", ctypes.c_int32), ("total_units", ctypes.c_int64),
        ("units", _i32p), ("unit_offset", _i64p), ("coupling_offset", _i64p), ("coupling", _dp),
        ("state", _dp), ("upar", _dp), ("uacc", _dp), ("iuacc", _i32p),
        ("time_domain", _dp), ("actual_time", _dp), ("rtol", _dp), ("atol", _dp),
        ("event_tol", ctypes.c_double), ("event_dir", ctypes.c_int32), ("algorithm", ctypes.c_int32),
        ("dt0", ctypes.c_double), ("dtmin", ctypes.c_double), ("dtmax", ctypes.c_double),
        ("grow", ctypes.c_double), ("shrink", ctypes.c_double),
        ("bicg_max_iter", ctypes.c_int32), ("shared_assoc", ctypes.c_int32), ("max_steps_per_period", ctypes.c_int64),
        ("ndo", ctypes.c_int32), ("do_save_frequency", ctypes.c_int32), ("do_min_dt", ctypes.c_double),
        ("dense_time", _dp), ("dense_state", _dp), ("dense_index", _i32p),
        ("n_accepted", _i64p), ("n_rejected", _i64p), ("n_bicg_iter", _i64p), ("n_rhs", _i64p),
        ("status", _i32p), ("coupling_row_scale", _dp), ("coupling_col_scale", _dp),
        ("bicg_variant", ctypes.c_int32), ("pad", ctypes.c_int32), ("min_dt", _dp),
        ("band_width", ctypes.c_int32), ("pad2", ctypes.c_int32),
    ]


def build(force: bool = False) -> Path:
    src = HERE / "bes_oracle.cpp"
    deps = [src, HERE / "bes_oracle.h", HERE / "oracle_math.h"]
    if force or not LIB.exists() or any(p.stat().st_mtime > LIB.stat().st_mtime for p in deps):
        cmd = ["g++", "-O3", "-std=c++17", "-ffp-contract=off", "-fopenmp", "-fPIC", "-shared",
               "-o", str(LIB), str(src)]
        subprocess.run(cmd, check=True)
    return LIB


_lib = None


def lib() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        build()
        L = ctypes.CDLL(str(LIB))
        L.bes_oracle_solve.argtypes = [ctypes.POINTER(Problem), ctypes.c_int, ctypes.c_int, _dp, _i32p, ctypes.c_int]
        L.bes_oracle_solve.restype = ctypes.c_int
        for n in ("bes_oracle_exp", "bes_oracle_log"):
            getattr(L, n).argtypes = [ctypes.c_double]
            getattr(L, n).restype = ctypes.c_double
        for n in ("bes_oracle_pow", "bes_oracle_pow_recip"):
            getattr(L, n).argtypes = [ctypes.c_double, ctypes.c_double]
            getattr(L, n).restype = ctypes.c_double
        L.bes_oracle_sincospi.argtypes = [ctypes.c_double, _dp, _dp]
        L.bes_oracle_sincos.argtypes = [ctypes.c_double, _dp, _dp]
        L.bes_oracle_rhs.argtypes = [ctypes.c_int, ctypes.c_double, _dp, _dp, _dp, ctypes.c_int, _dp]
        L.bes_oracle_rhs.restype = ctypes.c_int
        L.bes_oracle_max_threads.restype = ctypes.c_int
        L.bes_oracle_rec1_fallbacks.argtypes = [ctypes.c_int]
        L.bes_oracle_rec1_fallbacks.restype = ctypes.c_longlong
        L.bes_oracle_rec1_fallbacks_capped.argtypes = [ctypes.c_int]
        L.bes_oracle_rec1_fallbacks_capped.restype = ctypes.c_longlong
        _lib = L
    return _lib


def _p(a, t):
    return a.ctypes.data_as(t)


def run(ens, n_periods: int = None, reset_at: int = None, threads: int = 0, systems=None,
        algorithm: int = 1, ndo: int = 0, do_min_dt: float = 0.0, do_save_frequency: int = 1,
        bicg_max_iter: int = 19, uacc=None, iuacc=None, state=None, shared_assoc=None,
        bicg_variant: int = 0, band_width=None) -> dict:
    """Integrate an ``workloads.Ensemble`` on the CPU; returns the final arrays and counters."""
    if systems is not None:
        ens = ens.subset(systems)
    n_periods = ens.n_periods if n_periods is None else n_periods
    reset_at = ens.reset_at if reset_at is None else reset_at
    ns, tu = ens.n_systems, ens.total_units
    a = {
        "units": np.ascontiguousarray(ens.units, np.int32),
        "unit_offset": np.ascontiguousarray(ens.unit_offset, np.int64),
        "coupling_offset": np.ascontiguousarray(ens.coupling_offset(), np.int64),
        "coupling": np.ascontiguousarray(ens.coupling, np.float64),
        "state": np.ascontiguousarray(ens.state if state is None else state, np.float64).copy(),
        "upar": np.ascontiguousarray(ens.upar, np.float64),
        "uacc": np.ascontiguousarray(ens.initial_uacc() if uacc is None else uacc, np.float64).copy(),
        "iuacc": np.ascontiguousarray(ens.initial_iuacc() if iuacc is None else iuacc, np.int32).copy(),
        "time_domain": np.ascontiguousarray(np.stack([np.zeros(ns), np.ones(ns)]), np.float64),
        "actual_time": np.zeros(ns),
        "rtol": np.ascontiguousarray(ens.rtol, np.float64),
        "atol": np.ascontiguousarray(ens.atol, np.float64),
        "dense_time": np.zeros(max(1, ndo) * ns),
        "dense_state": np.zeros(max(1, ndo) * 2 * tu),
        "dense_index": np.zeros(ns, np.int32),
        "n_accepted": np.zeros(ns, np.int64), "n_rejected": np.zeros(ns, np.int64),
        "n_bicg_iter": np.zeros(ns, np.int64), "n_rhs": np.zeros(ns, np.int64),
        "status": np.zeros(ns, np.int32),
        "min_dt": np.full(ns, np.inf),
    }
    P = Problem()
    P.n_systems = ns
    P.active_systems = ns
    P.total_units = tu
    P.units = _p(a["units"], _i32p)
    P.unit_offset = _p(a["unit_offset"], _i64p)
    P.coupling_offset = _p(a["coupling_offset"], _i64p)
    for k in ("coupling", "state", "upar", "uacc", "time_domain", "actual_time", "rtol", "atol", "dense_time",
              "dense_state"):
        setattr(P, k, _p(a[k], _dp))
    P.iuacc = _p(a["iuacc"], _i32p)
    P.dense_index = _p(a["dense_index"], _i32p)
    for k in ("n_accepted", "n_rejected", "n_rhs"):
        setattr(P, k, _p(a[k], _i64p))
    P.n_bicg_iter = _p(a["n_bicg_iter"], _i64p)
    P.status = _p(a["status"], _i32p)
    P.event_tol = ens.event_tol
    P.event_dir = ens.event_dir
    P.algorithm = algorithm
    P.dt0, P.dtmin, P.dtmax, P.grow, P.shrink = ens.dt0, ens.dtmin, ens.dtmax, ens.grow, ens.shrink
    P.bicg_max_iter = bicg_max_iter
    P.bicg_variant = bicg_variant
    # banded coupling storage (the reference's CBW): the banded association where 2 bw + 1 < N
    P.band_width = int(getattr(ens, "band_width", 0) if band_width is None else band_width)
    P.min_dt = _p(a["min_dt"], _dp)
    # the library stages a launch's one shared matrix per CTA (and associates the products
    # accordingly) when the ensemble asks for shared coupling matrices
    P.shared_assoc = int(getattr(ens, "shared_matrices", False) if shared_assoc is None else shared_assoc)
    # per-unit coupling factors (a_i G_ij b_j) of a shared geometry, if the ensemble has them
    for k, attr in (("coupling_row_scale", "coupling_row_scale"), ("coupling_col_scale", "coupling_col_scale")):
        v = getattr(ens, attr, None)
        if v is not None:
            a[k] = np.ascontiguousarray(v, np.float64)
            setattr(P, k, _p(a[k], _dp))
    P.max_steps_per_period = ens.max_steps_per_period
    P.ndo = ndo
    P.do_save_frequency = do_save_frequency
    P.do_min_dt = do_min_dt
    ures = np.zeros(64)
    ires = np.array([-1], np.int32)
    rc = lib().bes_oracle_solve(ctypes.byref(P), n_periods, reset_at, _p(ures, _dp), _p(ires, _i32p), threads)
    if rc != 0:
        raise RuntimeError(f"oracle failed with {rc}")
    a["state"] = a["state"].reshape(2, tu)
    a["uacc"] = a["uacc"].reshape(64, tu)
    a["iuacc"] = a["iuacc"].reshape(1, tu)
    if ndo:
        a["dense_time"] = a["dense_time"].reshape(ndo, ns)
        a["dense_state"] = a["dense_state"].reshape(ndo, 2, tu)
    return a


def rhs(n: int, t: float, state: np.ndarray, upar: np.ndarray, coupling_colmajor: np.ndarray,
        bicg_max_iter: int = 19):
    """One coupled right-hand side of a single system (state [2, n], upar [21, n])."""
    s = np.ascontiguousarray(state, np.float64)
    u = np.ascontiguousarray(upar, np.float64)
    c = np.ascontiguousarray(coupling_colmajor, np.float64)
    f = np.zeros(2 * n)
    it = lib().bes_oracle_rhs(n, t, _p(s, _dp), _p(u, _dp), _p(c, _dp), bicg_max_iter, _p(f, _dp))
    return f.reshape(2, n), it


def max_threads() -> int:
    return lib().bes_oracle_max_threads()
