"""bes_solve_periods_noalloc: the solve for callers that cannot allocate device memory.

Such a caller (an application that owns the GPU's memory and hands out slices
of its own pool, or a loop where cudaMalloc could block) passes device
pointers of arrays it already holds; the entry point allocates nothing and
keeps the solver's scratch in a fixed device array inside the library.  This
test lays out an ensemble in device memory it allocates itself (with torch),
calls the entry point through the C ABI twice in a row, and checks both
results against the allocating entry point (bes_solve_periods via
ProblemSolver), bit for bit as the other parity tests do.  The file is named
to be collected last."""
import ctypes

import numpy as np
import pytest

from bubbleensemble_implicitextension_b200 import solver as S
from bubbleensemble_implicitextension_b200 import workloads as W
from tests.helpers import assert_bitwise, ragged_ensemble, run_gpu

pytestmark = pytest.mark.gpu
KEYS = ["state", "uacc", "iuacc", "n_accepted", "n_rejected", "n_bicg_iter", "n_rhs", "status"]


class DeviceEnsemble:
    """Every input and output array of an ensemble, in device memory owned by the caller."""

    def __init__(self, ens, ndo=0):
        import torch
        self.torch = torch
        dev = torch.device("cuda", 0)
        f64, i32, i64 = torch.float64, torch.int32, torch.int64
        self.ens = ens
        self.units_host = np.ascontiguousarray(ens.units, np.int32)
        t = lambda a, dt: torch.as_tensor(np.ascontiguousarray(a), dtype=dt, device=dev).contiguous()
        ns, tu = ens.n_systems, ens.total_units
        self.units = t(ens.units, i32)
        self.unit_offset = t(ens.unit_offset, i64)
        self.coupling_offset = t(ens.coupling_offset(), i64)
        self.coupling = t(ens.coupling, f64)
        self.upar = t(ens.upar, f64)
        self.rtol = t(ens.rtol, f64)
        self.atol = t(ens.atol, f64)
        self.event_tol = t([ens.event_tol], f64)
        self.event_dir = t([ens.event_dir], i32)
        self.uacc_reset = t(np.zeros(W.NUA), f64)
        self.iuacc_reset = t([-1], i32)
        td = np.zeros((2, ns))
        td[1] = 1.0
        self.time_domain = t(td, f64)
        self.state = torch.empty((2, tu), dtype=f64, device=dev)
        self.uacc = torch.empty((W.NUA, tu), dtype=f64, device=dev)
        self.iuacc = torch.empty((1, tu), dtype=i32, device=dev)
        self.actual_time = torch.empty(ns, dtype=f64, device=dev)
        self.cnt = torch.empty((4, ns), dtype=i64, device=dev)
        self.status = torch.empty(ns, dtype=i32, device=dev)
        self.ndo = ndo
        if ndo:
            self.dense_time = torch.empty((ndo, ns), dtype=f64, device=dev)
            self.dense_state = torch.empty((ndo, 2, tu), dtype=f64, device=dev)
            self.dense_index = torch.empty(ns, dtype=i32, device=dev)
        self.errbuf = ctypes.create_string_buffer(512)

    def reset(self):
        ens, torch = self.ens, self.torch
        self.state.copy_(torch.as_tensor(ens.state))
        self.uacc.copy_(torch.as_tensor(ens.initial_uacc()))
        self.iuacc.copy_(torch.as_tensor(ens.initial_iuacc()))
        self.actual_time.zero_()
        self.cnt.zero_()
        self.status.zero_()
        if self.ndo:
            self.dense_time.zero_()
            self.dense_state.zero_()
            self.dense_index.zero_()
        torch.cuda.synchronize()

    def problem(self, algorithm=S.Algorithms.RKCK45, do_min_dt=0.0, do_save_frequency=1, options=True,
                bicg_recurrence=0):
        ens = self.ens
        p = S.NoallocProblem()
        p.n_systems = ens.n_systems
        p.algorithm = algorithm
        p.total_units = ens.total_units
        p.units_host = self.units_host.ctypes.data_as(ctypes.POINTER(ctypes.c_int32))
        for name in ("units", "unit_offset", "coupling_offset", "coupling", "state", "upar", "uacc", "iuacc",
                     "time_domain", "actual_time", "rtol", "atol", "event_tol", "event_dir", "uacc_reset",
                     "iuacc_reset", "status"):
            setattr(p, name, getattr(self, name).data_ptr())
        base, step = self.cnt.data_ptr(), self.cnt.stride(0) * 8
        p.n_accepted, p.n_rejected, p.n_bicg_iter, p.n_rhs = base, base + step, base + 2 * step, base + 3 * step
        if self.ndo:
            for name in ("dense_time", "dense_state", "dense_index"):
                setattr(p, name, getattr(self, name).data_ptr())
            p.ndo, p.do_min_dt, p.do_save_frequency = self.ndo, do_min_dt, do_save_frequency
        if options:   # otherwise left 0: the SolverOption defaults
            p.dt0, p.dtmin, p.dtmax, p.grow, p.shrink = ens.dt0, ens.dtmin, ens.dtmax, ens.grow, ens.shrink
            p.bicg_max_iter = 19
        p.max_steps_per_period = ens.max_steps_per_period
        p.bicg_recurrence = bicg_recurrence
        p.error_message = ctypes.cast(self.errbuf, ctypes.c_char_p)
        p.error_capacity = len(self.errbuf)
        return p

    def results(self):
        self.torch.cuda.synchronize()
        c = self.cnt.cpu().numpy()
        out = {"state": self.state.cpu().numpy(), "uacc": self.uacc.cpu().numpy(), "iuacc": self.iuacc.cpu().numpy(),
               "n_accepted": c[0], "n_rejected": c[1], "n_bicg_iter": c[2], "n_rhs": c[3],
               "status": self.status.cpu().numpy()}
        if self.ndo:
            out.update({"dense_time": self.dense_time.cpu().numpy(), "dense_state": self.dense_state.cpu().numpy(),
                        "dense_index": self.dense_index.cpu().numpy()})
        return out


def _bounded(ens):
    ens.max_steps_per_period = 50_000
    return ens


@pytest.mark.parametrize("case", ["c1_uniform32", "ragged"])
def test_noalloc_matches_allocating_entry_point_twice(case, gpu):
    lib = S.load_library()
    if case == "c1_uniform32":
        ens = _bounded(W.c1_ensemble().subset([1, 50, 99, 160, 230]))
    else:
        ens = _bounded(ragged_ensemble([32, 16, 48, 8, 64, 31], seed=21))
    want = run_gpu(ens, n_periods=2, reset_at=1)
    dev = DeviceEnsemble(ens)
    for call in range(2):
        dev.reset()
        p = dev.problem()
        st = lib.bes_solve_periods_noalloc(ctypes.byref(p), 2, 1, None)
        assert st == 0, dev.errbuf.value.decode()
        assert_bitwise(dev.results(), want, KEYS)


def test_noalloc_rejects_more_systems_than_its_scratch(gpu):
    lib = S.load_library()
    p = S.NoallocProblem()
    p.n_systems = 65537
    buf = ctypes.create_string_buffer(256)
    p.error_message = ctypes.cast(buf, ctypes.c_char_p)
    p.error_capacity = 256
    assert lib.bes_solve_periods_noalloc(ctypes.byref(p), 1, -1, None) == 1
    assert b"65536" in buf.value


def test_noalloc_zero_options_take_the_solver_option_defaults(gpu):
    """dt0, dtmin, dtmax, grow, shrink and the BiCG cap left 0 mean the reference's
    SolverOption defaults (Interface.cuh:613-618): the allocating entry point with
    those defaults set gives the same results."""
    lib = S.load_library()
    ens = _bounded(W.c1_ensemble().subset([12, 140]))
    ens.dt0, ens.dtmin, ens.dtmax, ens.grow, ens.shrink = 1e-2, 1e-12, 1e6, 5.0, 0.1
    want = run_gpu(ens, n_periods=1, reset_at=-1)
    dev = DeviceEnsemble(ens)
    for call in range(2):
        dev.reset()
        p = dev.problem(options=False)
        st = lib.bes_solve_periods_noalloc(ctypes.byref(p), 1, -1, None)
        assert st == 0, dev.errbuf.value.decode()
        assert_bitwise(dev.results(), want, KEYS)


def test_noalloc_rejects_negative_options(gpu):
    lib = S.load_library()
    ens = _bounded(W.c1_ensemble().subset([3]))
    dev = DeviceEnsemble(ens)
    dev.reset()
    p = dev.problem()
    p.dtmax = -1.0
    assert lib.bes_solve_periods_noalloc(ctypes.byref(p), 1, -1, None) == 1
    assert b"dtmax" in dev.errbuf.value


def test_noalloc_dense_output_rk4_on_a_caller_stream(gpu):
    """Dense output and the RK4 stepper, launched on a stream the caller created."""
    import torch
    lib = S.load_library()
    ens = _bounded(W.c1_ensemble().subset([40, 41, 200]))
    ens.dt0 = 2e-3
    want = run_gpu(ens, n_periods=2, reset_at=-1, algorithm=S.Algorithms.RK4, ndo=16, do_min_dt=0.05,
                   do_save_frequency=2)
    dev = DeviceEnsemble(ens, ndo=16)
    stream = torch.cuda.Stream()
    for call in range(2):
        dev.reset()
        p = dev.problem(algorithm=S.Algorithms.RK4, do_min_dt=0.05, do_save_frequency=2)
        st = lib.bes_solve_periods_noalloc(ctypes.byref(p), 2, -1, ctypes.c_void_p(stream.cuda_stream))
        assert st == 0, dev.errbuf.value.decode()
        stream.synchronize()
        assert_bitwise(dev.results(), want, KEYS + ["dense_time", "dense_state", "dense_index"])


def test_noalloc_single_reduction_recurrence(gpu):
    lib = S.load_library()
    ens = _bounded(ragged_ensemble([32, 64, 20, 128], seed=23))
    want = run_gpu(ens, n_periods=1, reset_at=-1, bicg_recurrence=1)
    dev = DeviceEnsemble(ens)
    for call in range(2):
        dev.reset()
        p = dev.problem(bicg_recurrence=1)
        st = lib.bes_solve_periods_noalloc(ctypes.byref(p), 1, -1, None)
        assert st == 0, dev.errbuf.value.decode()
        assert_bitwise(dev.results(), want, KEYS)
