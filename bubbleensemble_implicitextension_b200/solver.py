"""ctypes binding of ``libbes.so`` that mirrors the reference's ``ProblemSolver``.

The reference's host API is the C++ class template ``ProblemSolver<...>``
(SourceCodes/CoupledSystems_PerBlock_Interface.cuh:135-248).  This module
keeps its member names (``SolverOption``, ``SetHost``, ``GetHost``,
``SynchroniseFromHostToDevice``, ``SynchroniseFromDeviceToHost``, ``Solve``,
``InsertSynchronisationPoint``, ``SynchroniseSolver``, ``SynchroniseDevice``),
its enumerations (``ListOfVariables``, ``ListOfSolverOptions``,
``Algorithms``) and the argument meaning of every overload.  Errors that
make the reference call ``exit()`` raise :class:`BesError` here.

The library is the only compute path: if ``libbes.so`` is missing or cannot
be loaded, importing this module's ``load_library`` raises; there is no CPU
fallback.
"""
from __future__ import annotations

import ctypes
import os
from pathlib import Path
from typing import Optional, Sequence

import numpy as np
from enum import IntEnum

class ListOfVariables(IntEnum):
    """Interface.cuh:35-53 (same order), plus extensions from 100 on."""
    All = 0
    TimeDomain = 1
    ActualTime = 2
    ActualState = 3
    UnitParameters = 4
    SystemParameters = 5
    GlobalParameters = 6
    IntegerGlobalParameters = 7
    UnitAccessories = 8
    IntegerUnitAccessories = 9
    SystemAccessories = 10
    IntegerSystemAccessories = 11
    CouplingMatrix = 12
    CouplingStrength = 13
    CouplingIndex = 14
    DenseOutput = 15
    DenseIndex = 16
    DenseTime = 17
    DenseState = 18
    RelativeToleranceSystem = 100
    AbsoluteToleranceSystem = 101
    Counters = 102
    CouplingRowScale = 103
    CouplingColumnScale = 104
    PoincareSections = 105
    PeriodNumber = 106
    MaximumAccessory = 107


class ListOfSolverOptions(IntEnum):
    """Interface.cuh:55-68 (same order), plus extensions from 100 on."""
    InitialTimeStep = 0
    ActiveSystems = 1
    MaximumTimeStep = 2
    MinimumTimeStep = 3
    TimeStepGrowLimit = 4
    TimeStepShrinkLimit = 5
    RelativeTolerance = 6
    AbsoluteTolerance = 7
    EventTolerance = 8
    EventDirection = 9
    DenseOutputSaveFrequency = 10
    DenseOutputMinimumTimeStep = 11
    SharedGlobalVariables = 12
    SharedCouplingMatrices = 13
    MaxStepsPerPeriod = 100
    BiCGMaxIterations = 101
    WarpsPerBlock = 102
    UseCudaGraph = 103
    WarpsPerSystem = 104
    BiCGRecurrence = 105


class Algorithms(IntEnum):
    """Interface.cuh:33"""
    RK4 = 0
    RKCK45 = 1


globals().update({m.name: m for m in ListOfVariables})
globals().update({m.name: m for m in ListOfSolverOptions})
globals().update({m.name: m for m in Algorithms})

STATUS_NONFINITE = 1
STATUS_MIN_STEP = 2
STATUS_STEP_BUDGET = 4
STATUS_EVENT_MISSED = 8
STATUS_BICG_CAP = 16

_INT_VARS = {ListOfVariables.IntegerGlobalParameters, ListOfVariables.IntegerUnitAccessories,
             ListOfVariables.IntegerSystemAccessories, ListOfVariables.CouplingIndex, ListOfVariables.DenseIndex,
             ListOfVariables.PeriodNumber}

LIB_PATH = Path(__file__).resolve().parent / "libbes.so"


class BesError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"[bes status {status}] {message}")
        self.status = status


class _Config(ctypes.Structure):
    _fields_ = [
        ("device", ctypes.c_int32), ("n_systems", ctypes.c_int32), ("units_per_system", ctypes.c_int32),
        ("units", ctypes.POINTER(ctypes.c_int32)),
        ("unit_dim", ctypes.c_int32), ("n_unit_parameters", ctypes.c_int32), ("n_system_parameters", ctypes.c_int32),
        ("n_global_parameters", ctypes.c_int32), ("n_int_global_parameters", ctypes.c_int32),
        ("n_unit_accessories", ctypes.c_int32), ("n_int_unit_accessories", ctypes.c_int32),
        ("n_system_accessories", ctypes.c_int32), ("n_int_system_accessories", ctypes.c_int32),
        ("n_events", ctypes.c_int32), ("n_dense_output", ctypes.c_int32), ("n_couplings", ctypes.c_int32),
        ("coupling_bandwidth", ctypes.c_int32), ("coupling_circular", ctypes.c_int32),
        ("algorithm", ctypes.c_int32), ("n_coupling_matrices", ctypes.c_int32),
        ("coupling_matrix_of_system", ctypes.POINTER(ctypes.c_int32)),
    ]


class ModelInfo(ctypes.Structure):
    _fields_ = [
        ("unit_dim", ctypes.c_int32), ("n_unit_parameters", ctypes.c_int32),
        ("n_system_parameters", ctypes.c_int32), ("n_global_parameters", ctypes.c_int32),
        ("n_int_global_parameters", ctypes.c_int32), ("n_unit_accessories", ctypes.c_int32),
        ("n_int_unit_accessories", ctypes.c_int32), ("n_system_accessories", ctypes.c_int32),
        ("n_int_system_accessories", ctypes.c_int32), ("n_events", ctypes.c_int32),
        ("max_units_per_system", ctypes.c_int32), ("name", ctypes.c_char * 64),
    ]


class DeviceInfo(ctypes.Structure):
    _fields_ = [("name", ctypes.c_char * 256), ("cc_major", ctypes.c_int32), ("cc_minor", ctypes.c_int32),
                ("multiprocessors", ctypes.c_int32), ("pad", ctypes.c_int32), ("global_memory_bytes", ctypes.c_uint64)]


class CountersStruct(ctypes.Structure):
    _fields_ = [
        ("accepted_steps", ctypes.c_uint64), ("rejected_steps", ctypes.c_uint64),
        ("bicg_iterations", ctypes.c_uint64), ("rhs_evaluations", ctypes.c_uint64),
        ("status", ctypes.c_int32), ("units", ctypes.c_int32),
    ]


class CsvKind(IntEnum):
    """bes_write_csv kinds: the reference drivers' output files."""
    Collapse = 0     # CollapseStrength.cu:174-198
    Poincare = 1     # BubbleEnsemble.cu:435-455
    Period = 2       # BubbleEnsemble.cu:457-473
    Expansion = 3    # BubbleEnsemble.cu:475-491


class AutotuneResult(ctypes.Structure):
    _fields_ = [("warps_per_block", ctypes.c_int32 * 3), ("warps_per_system", ctypes.c_int32 * 3),
                ("ms", ctypes.c_float * 3), ("candidates", ctypes.c_int32)]


class MlpConfig(ctypes.Structure):
    _fields_ = [("device", ctypes.c_int32), ("n_in", ctypes.c_int32), ("width", ctypes.c_int32),
                ("depth", ctypes.c_int32), ("n_out", ctypes.c_int32), ("max_batch", ctypes.c_int32),
                ("seed", ctypes.c_uint64)]


class NoallocProblem(ctypes.Structure):
    """bes_noalloc_problem (include/bes.h): device pointers of a caller-owned ensemble."""
    _P64 = ctypes.c_void_p
    _fields_ = [
        ("n_systems", ctypes.c_int32), ("algorithm", ctypes.c_int32), ("total_units", ctypes.c_int64),
        ("units_host", ctypes.POINTER(ctypes.c_int32)),
        ("units", _P64), ("unit_offset", _P64), ("coupling_offset", _P64), ("coupling", _P64),
        ("state", _P64), ("upar", _P64), ("uacc", _P64), ("iuacc", _P64),
        ("spar", _P64), ("sacc", _P64), ("isacc", _P64), ("gpar", _P64), ("igpar", _P64),
        ("time_domain", _P64), ("actual_time", _P64), ("rtol", _P64), ("atol", _P64),
        ("event_tol", _P64), ("event_dir", _P64), ("uacc_reset", _P64), ("iuacc_reset", _P64),
        ("dense_time", _P64), ("dense_state", _P64), ("dense_index", _P64),
        ("n_accepted", _P64), ("n_rejected", _P64), ("n_bicg_iter", _P64), ("n_rhs", _P64), ("status", _P64),
        ("dt0", ctypes.c_double), ("dtmin", ctypes.c_double), ("dtmax", ctypes.c_double),
        ("grow", ctypes.c_double), ("shrink", ctypes.c_double), ("do_min_dt", ctypes.c_double),
        ("ndo", ctypes.c_int32), ("do_save_frequency", ctypes.c_int32),
        ("bicg_max_iter", ctypes.c_int32), ("warps_per_block", ctypes.c_int32),
        ("max_steps_per_period", ctypes.c_int64),
        ("error_message", ctypes.c_char_p), ("error_capacity", ctypes.c_int32), ("bicg_recurrence", ctypes.c_int32),
    ]


# every exported symbol of include/bes.h with its argument types
_I32, _D, _P = ctypes.c_int32, ctypes.c_double, ctypes.c_void_p
_DP = ctypes.POINTER(ctypes.c_double)
SIGNATURES = {
    "bes_autotune": [_P, _I32, ctypes.c_int64, ctypes.POINTER(AutotuneResult)],
    "bes_set_period_analysis": [_P, _I32, _D, _I32],
    "bes_write_csv": [_P, _I32, ctypes.c_char_p],
    "bes_print": [_P, _I32, _I32, ctypes.c_char_p],
    "bes_create": [ctypes.POINTER(_Config), ctypes.POINTER(ctypes.c_void_p)],
    "bes_destroy": [_P],
    "bes_model_info_get": [ctypes.POINTER(ModelInfo)],
    "bes_solver_option": [_P, _I32, _D],
    "bes_solver_option_indexed": [_P, _I32, _I32, _D],
    "bes_set_host_unit": [_P, _I32, _I32, _I32, _I32, _D],
    "bes_set_host_system": [_P, _I32, _I32, _I32, _D],
    "bes_set_host_global": [_P, _I32, _I32, _D],
    "bes_set_host_coupling": [_P, _I32, _I32, _I32, _I32, _D],
    "bes_set_host_dense_index": [_P, _I32, _I32, _D],
    "bes_set_host_dense_state": [_P, _I32, _I32, _I32, _I32, _I32, _D],
    "bes_get_host_unit": [_P, _I32, _I32, _I32, _I32, _DP],
    "bes_get_host_system": [_P, _I32, _I32, _I32, _DP],
    "bes_get_host_global": [_P, _I32, _I32, _DP],
    "bes_get_host_coupling": [_P, _I32, _I32, _I32, _I32, _DP],
    "bes_get_host_dense_index": [_P, _I32, _I32, _DP],
    "bes_get_host_dense_state": [_P, _I32, _I32, _I32, _I32, _I32, _DP],
    "bes_set_array": [_P, _I32, _P, ctypes.c_int64],
    "bes_get_array": [_P, _I32, _P, ctypes.c_int64],
    "bes_array_size": [_P, _I32, ctypes.POINTER(ctypes.c_int64)],
    "bes_synchronise_host_to_device": [_P, _I32],
    "bes_synchronise_device_to_host": [_P, _I32],
    "bes_solve": [_P],
    "bes_solve_periods": [_P, _I32, _I32],
    "bes_set_accessory_reset": [_P, _DP, ctypes.POINTER(ctypes.c_int32)],
    "bes_synchronise_device": [_P],
    "bes_insert_synchronisation_point": [_P],
    "bes_synchronise_solver": [_P],
    "bes_set_stream": [_P, _P],
    "bes_last_solve_ms": [_P, ctypes.POINTER(ctypes.c_float)],
    "bes_last_solve_launches": [_P, ctypes.POINTER(ctypes.c_int32)],
    "bes_get_counters": [_P, _I32, ctypes.POINTER(CountersStruct)],
    "bes_reset_counters": [_P],
    "bes_load_bubble_sizes": [ctypes.c_char_p, _I32, _DP],
    "bes_load_coupling_matrix": [ctypes.c_char_p, _I32, _DP],
    "bes_device_count": [ctypes.POINTER(ctypes.c_int32)],
    "bes_device_info_get": [_I32, ctypes.POINTER(DeviceInfo)],
    "bes_measure_fp64_peak": [_I32, ctypes.POINTER(ctypes.c_double)],
    "bes_solve_periods_noalloc": [ctypes.POINTER(NoallocProblem), _I32, _I32, _P],
    "bes_mlp_create": [ctypes.POINTER(MlpConfig), ctypes.POINTER(ctypes.c_void_p)],
    "bes_mlp_destroy": [_P],
    "bes_mlp_parameter_count": [_P, ctypes.POINTER(ctypes.c_int64)],
    "bes_mlp_set_normalization": [_P, ctypes.POINTER(ctypes.c_float), ctypes.POINTER(ctypes.c_float),
                                  ctypes.POINTER(ctypes.c_float), ctypes.POINTER(ctypes.c_float)],
    "bes_mlp_get_parameters": [_P, ctypes.POINTER(ctypes.c_float), ctypes.c_int64],
    "bes_mlp_set_parameters": [_P, ctypes.POINTER(ctypes.c_float), ctypes.c_int64],
    "bes_mlp_get_gradients": [_P, ctypes.POINTER(ctypes.c_float), ctypes.c_int64],
    "bes_mlp_forward": [_P, _P, _I32, _P, _P],
    "bes_mlp_backward": [_P, _P, _P, _I32, ctypes.POINTER(ctypes.c_float), _P],
    "bes_mlp_adam_step": [_P, ctypes.c_float, _P],
    "bes_mlp_last_error": [_P],
    "bes_status_string": [_I32],
    "bes_last_error": [_P],
}

_lib: Optional[ctypes.CDLL] = None


def load_library(path: Optional[os.PathLike] = None) -> ctypes.CDLL:
    """Load ``libbes.so`` and declare every entry point.  Raises when absent."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = Path(path) if path is not None else LIB_PATH
    if not p.exists():
        raise BesError(-1, f"{p} is missing: build it with bubbleensemble_implicitextension_b200._build.build()")
    lib = ctypes.CDLL(str(p))
    for name, args in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.argtypes = args
        fn.restype = (ctypes.c_char_p if name in ("bes_status_string", "bes_last_error", "bes_mlp_last_error")
                      else ctypes.c_int32)
    if path is None:
        _lib = lib
    return lib


def model_info() -> ModelInfo:
    lib = load_library()
    info = ModelInfo()
    _check(lib, None, lib.bes_model_info_get(ctypes.byref(info)))
    return info


def device_count() -> int:
    lib = load_library()
    n = ctypes.c_int32(0)
    st = lib.bes_device_count(ctypes.byref(n))
    return n.value if st == 0 else 0


def measure_fp64_peak(device: int = 0) -> float:
    """FP64 FMA throughput of the device in TFLOP/s (bes_measure_fp64_peak)."""
    lib = load_library()
    t = ctypes.c_double()
    _check(lib, None, lib.bes_measure_fp64_peak(device, ctypes.byref(t)))
    return t.value


def _check(lib, handle, status: int) -> None:
    if status != 0:
        msg = lib.bes_last_error(handle).decode(errors="replace") if lib is not None else ""
        raise BesError(status, msg or lib.bes_status_string(status).decode())


def load_bubble_sizes(path: os.PathLike, n: int) -> np.ndarray:
    """LoadBubbleSizes (CollapseStrength.cu:245-258) through the library."""
    lib = load_library()
    out = np.zeros(n, dtype=np.float64)
    _check(lib, None, lib.bes_load_bubble_sizes(os.fsencode(path), n, out.ctypes.data_as(_DP)))
    return out


def load_coupling_matrix(path: os.PathLike, n: int) -> np.ndarray:
    """LoadCouplingMatrix (CollapseStrength.cu:260-277): returns M[row, col]."""
    lib = load_library()
    out = np.zeros(n * n, dtype=np.float64)
    _check(lib, None, lib.bes_load_coupling_matrix(os.fsencode(path), n, out.ctypes.data_as(_DP)))
    return out.reshape(n, n)


class ProblemSolver:
    """One solver object: the reference's ``ProblemSolver`` with run-time sizes.

    ``units`` is either an int (every system has that many units, the
    reference's UPS) or a sequence with one count per system.
    """

    def __init__(self, n_systems: int, units, *, algorithm: int = Algorithms.RKCK45, n_dense_output: int = 0,
                 n_couplings: int = 1, n_coupling_matrices: int = 1,
                 coupling_matrix_of_system: Optional[Sequence[int]] = None, device: int = 0,
                 model: Optional[ModelInfo] = None, library: Optional[os.PathLike] = None,
                 coupling_bandwidth: int = 0, coupling_circular: int = 0):
        self._lib = load_library(library)
        info = ModelInfo()
        _check(self._lib, None, self._lib.bes_model_info_get(ctypes.byref(info)))
        m = model or info
        cfg = _Config()
        cfg.device = device
        cfg.n_systems = n_systems
        self._units_arr = None
        if isinstance(units, (int, np.integer)):
            cfg.units_per_system = int(units)
            self.units = np.full(n_systems, int(units), dtype=np.int32)
        else:
            self._units_arr = np.ascontiguousarray(units, dtype=np.int32)
            if self._units_arr.shape != (n_systems,):
                raise ValueError("units must have one entry per system")
            cfg.units_per_system = 0
            cfg.units = self._units_arr.ctypes.data_as(ctypes.POINTER(ctypes.c_int32))
            self.units = self._units_arr.copy()
        for f in ("unit_dim", "n_unit_parameters", "n_system_parameters", "n_global_parameters",
                  "n_int_global_parameters", "n_unit_accessories", "n_int_unit_accessories",
                  "n_system_accessories", "n_int_system_accessories", "n_events"):
            setattr(cfg, f, getattr(m, f))
        cfg.n_dense_output = n_dense_output
        cfg.coupling_bandwidth = coupling_bandwidth
        cfg.coupling_circular = coupling_circular
        cfg.n_couplings = n_couplings
        cfg.algorithm = algorithm
        cfg.n_coupling_matrices = n_coupling_matrices
        self._mos = None
        if coupling_matrix_of_system is not None:
            self._mos = np.ascontiguousarray(coupling_matrix_of_system, dtype=np.int32)
            cfg.coupling_matrix_of_system = self._mos.ctypes.data_as(ctypes.POINTER(ctypes.c_int32))
        h = ctypes.c_void_p()
        _check(self._lib, None, self._lib.bes_create(ctypes.byref(cfg), ctypes.byref(h)))
        self._h = h
        self.n_systems = n_systems
        self.model = info
        self.n_dense_output = n_dense_output
        self.unit_offset = np.concatenate([[0], np.cumsum(self.units)[:-1]]).astype(np.int64)
        self.total_units = int(self.units.sum())

    # -- lifetime ---------------------------------------------------------------------
    def close(self) -> None:
        if getattr(self, "_h", None):
            self._lib.bes_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def _ok(self, status: int) -> None:
        _check(self._lib, self._h, status)

    # -- options (Interface.cuh:774-865) ------------------------------------------------
    def SolverOption(self, option: int, *args) -> None:
        if len(args) == 1:
            self._ok(self._lib.bes_solver_option(self._h, option, float(args[0])))
        elif len(args) == 2:
            self._ok(self._lib.bes_solver_option_indexed(self._h, option, int(args[0]), float(args[1])))
        else:
            raise TypeError("SolverOption(option, value) or SolverOption(option, index, value)")

    # -- element access (Interface.cuh:870-1140, :1341-1529) ---------------------------
    def SetHost(self, *args) -> None:
        """Overloads by argument list, as in the reference (variables must be
        ``ListOfVariables`` members, which is what tells the overloads apart):
        (sid, uid, var, k, v) unit scope; (sid, var, k, v) system scope / dense time;
        (var, k, v) global scope; (n, CouplingMatrix, row, col, v) coupling;
        (sid, DenseIndex, v) dense index; (sid, uid, DenseState, comp, slot, v) dense state."""
        L = self._lib
        if len(args) == 6:
            sid, uid, var, comp, slot, v = args
            st = L.bes_set_host_dense_state(self._h, sid, uid, var, comp, slot, float(v))
        elif len(args) == 5:
            if isinstance(args[1], ListOfVariables):
                n, var, row, col, v = args
                st = L.bes_set_host_coupling(self._h, n, var, row, col, float(v))
            else:
                sid, uid, var, k, v = args
                st = L.bes_set_host_unit(self._h, sid, uid, var, k, float(v))
        elif len(args) == 4:
            sid, var, k, v = args
            st = L.bes_set_host_system(self._h, sid, var, k, float(v))
        elif len(args) == 3:
            if isinstance(args[0], ListOfVariables):
                var, k, v = args
                st = L.bes_set_host_global(self._h, var, k, float(v))
            else:
                sid, var, v = args
                st = L.bes_set_host_dense_index(self._h, sid, var, float(v))
        else:
            raise TypeError("SetHost: unsupported argument list")
        self._ok(st)

    def GetHost(self, *args) -> float:
        L = self._lib
        out = ctypes.c_double()
        ref = ctypes.byref(out)
        if len(args) == 5:
            sid, uid, var, comp, slot = args
            st = L.bes_get_host_dense_state(self._h, sid, uid, var, comp, slot, ref)
        elif len(args) == 4:
            if isinstance(args[1], ListOfVariables):
                n, var, row, col = args
                st = L.bes_get_host_coupling(self._h, n, var, row, col, ref)
            else:
                sid, uid, var, k = args
                st = L.bes_get_host_unit(self._h, sid, uid, var, k, ref)
        elif len(args) == 3:
            sid, var, k = args
            st = L.bes_get_host_system(self._h, sid, var, k, ref)
        elif len(args) == 2:
            if isinstance(args[0], ListOfVariables):
                var, k = args
                st = L.bes_get_host_global(self._h, var, k, ref)
            else:
                sid, var = args
                st = L.bes_get_host_dense_index(self._h, sid, var, ref)
        else:
            raise TypeError("GetHost: unsupported argument list")
        self._ok(st)
        return out.value

    # -- bulk access (extension) -------------------------------------------------------
    def array_size(self, var: int) -> int:
        n = ctypes.c_int64()
        self._ok(self._lib.bes_array_size(self._h, var, ctypes.byref(n)))
        return n.value

    def set_array(self, var: int, values) -> None:
        dt = np.int32 if var in _INT_VARS else np.float64
        a = np.ascontiguousarray(values, dtype=dt).ravel()
        self._ok(self._lib.bes_set_array(self._h, var, a.ctypes.data, a.size))

    def get_array(self, var: int) -> np.ndarray:
        dt = np.int32 if var in _INT_VARS else np.float64
        a = np.empty(self.array_size(var), dtype=dt)
        self._ok(self._lib.bes_get_array(self._h, var, a.ctypes.data, a.size))
        return a

    # -- transfers (Interface.cuh:1144-1336) -------------------------------------------
    def SynchroniseFromHostToDevice(self, var: int) -> None:
        self._ok(self._lib.bes_synchronise_host_to_device(self._h, var))

    def SynchroniseFromDeviceToHost(self, var: int) -> None:
        self._ok(self._lib.bes_synchronise_device_to_host(self._h, var))

    # -- execution (Interface.cuh:1951-1983) -------------------------------------------
    def Solve(self) -> None:
        self._ok(self._lib.bes_solve(self._h))

    def solve_periods(self, n_periods: int, reset_at: int = -1) -> None:
        self._ok(self._lib.bes_solve_periods(self._h, n_periods, reset_at))

    def set_accessory_reset(self, uacc, iuacc) -> None:
        u = np.ascontiguousarray(uacc, dtype=np.float64)
        i = np.ascontiguousarray(iuacc, dtype=np.int32)
        self._ok(self._lib.bes_set_accessory_reset(self._h, u.ctypes.data_as(_DP),
                                                   i.ctypes.data_as(ctypes.POINTER(ctypes.c_int32))))

    def SynchroniseDevice(self) -> None:
        self._ok(self._lib.bes_synchronise_device(self._h))

    def InsertSynchronisationPoint(self) -> None:
        self._ok(self._lib.bes_insert_synchronisation_point(self._h))

    def SynchroniseSolver(self) -> None:
        self._ok(self._lib.bes_synchronise_solver(self._h))

    def set_stream(self, cuda_stream_ptr: int) -> None:
        self._ok(self._lib.bes_set_stream(self._h, ctypes.c_void_p(cuda_stream_ptr)))

    def last_solve_ms(self) -> float:
        ms = ctypes.c_float()
        self._ok(self._lib.bes_last_solve_ms(self._h, ctypes.byref(ms)))
        return ms.value

    def set_period_analysis(self, sections: int, distance_tolerance: float = 1e-6, accessory_index: int = 0) -> None:
        """Per-period analysis of the following solves on the device (bes_set_period_analysis);
        sections < 0 turns it off."""
        self._ok(self._lib.bes_set_period_analysis(self._h, sections, distance_tolerance, accessory_index))

    def Print(self, var: int, serial: int = 0, directory=None) -> None:
        """Print(var) / Print(var, n) of the reference (bes_print): the host mirror to a text file."""
        d = None if directory is None else str(directory).encode()
        self._ok(self._lib.bes_print(self._h, var, serial, d))

    def write_csv(self, kind: int, path) -> None:
        """One of the reference drivers' output files from the host mirrors (bes_write_csv)."""
        self._ok(self._lib.bes_write_csv(self._h, kind, str(path).encode()))

    def autotune(self, n_periods: int = 1, step_cap: int = 2000) -> dict:
        """Time every launch shape per size class on the device's current inputs
        and keep the fastest (bes_autotune); the device state is restored."""
        r = AutotuneResult()
        self._ok(self._lib.bes_autotune(self._h, n_periods, step_cap, ctypes.byref(r)))
        return {"warps_per_block": list(r.warps_per_block), "warps_per_system": list(r.warps_per_system),
                "ms": [float(x) for x in r.ms], "candidates": int(r.candidates)}

    def last_solve_launches(self) -> int:
        n = ctypes.c_int32()
        self._ok(self._lib.bes_last_solve_launches(self._h, ctypes.byref(n)))
        return n.value

    def reset_counters(self) -> None:
        self._ok(self._lib.bes_reset_counters(self._h))

    def counters(self) -> dict:
        """Per-system counters from the host mirror (after D2H of ``Counters``)."""
        c = CountersStruct()
        acc = np.zeros(self.n_systems, np.uint64)
        rej = np.zeros_like(acc)
        bicg = np.zeros_like(acc)
        rhs = np.zeros_like(acc)
        status = np.zeros(self.n_systems, np.int32)
        for s in range(self.n_systems):
            self._ok(self._lib.bes_get_counters(self._h, s, ctypes.byref(c)))
            acc[s], rej[s], bicg[s], rhs[s], status[s] = (c.accepted_steps, c.rejected_steps, c.bicg_iterations,
                                                          c.rhs_evaluations, c.status)
        return {"accepted": acc, "rejected": rej, "bicg": bicg, "rhs": rhs, "status": status}
