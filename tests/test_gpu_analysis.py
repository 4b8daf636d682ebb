"""Per-period analysis on the device (Poincare sections, period detection,
running accessory maximum; BubbleEnsemble.cu:174-216) against the oracle run
period by period, and the reference drivers' output files (bes_write_csv)."""
import numpy as np
import pytest

from bubbleensemble_implicitextension_b200 import solver as S
from bubbleensemble_implicitextension_b200 import workloads as W

pytestmark = pytest.mark.gpu
V = S.ListOfVariables


def _ensemble():
    ens = W.c1_ensemble().subset([0, 17, 34, 51, 100])   # low to mid amplitude, several frequencies
    ens.max_steps_per_period = 50_000
    return ens


def _oracle_analysis(oracle_lib, ens, state0, uacc0, iuacc0, n_periods, tol, acc):
    """The same quantities from the oracle, one reference Solve() per period."""
    tu = ens.total_units
    state, uacc, iuacc = state0.copy(), uacc0.copy(), iuacc0.copy()
    sections = np.zeros((n_periods, tu))
    period = np.zeros(tu, np.int32)
    mx = uacc0[acc].copy()
    for p in range(n_periods):
        out = oracle_lib.run(ens, n_periods=1, reset_at=-1, state=state, uacc=uacc, iuacc=iuacc)
        state, uacc, iuacc = out["state"].reshape(2, -1), out["uacc"].reshape(64, -1), out["iuacc"].reshape(1, -1)
        sections[p] = state[0]
        d0, d1 = state0[0] - state[0], state0[1] - state[1]
        hit = (np.sqrt(d0 * d0 + d1 * d1) < tol) & (period == 0)
        period[hit] = p + 1
        mx = np.where(uacc[acc] > mx, uacc[acc], mx)
    return sections, period, mx, state


def test_period_analysis_matches_oracle(gpu, oracle_lib, tmp_path):
    ens = _ensemble()
    n_tr, n_an, tol = 1, 4, 2e-2
    ps = ens.make_solver()
    try:
        ps.SynchroniseFromHostToDevice(V.All)
        ps.solve_periods(n_tr, -1)                      # transient, analysis off
        ps.SynchroniseFromDeviceToHost(V.All)
        ps.InsertSynchronisationPoint()
        ps.SynchroniseSolver()
        state0 = ps.get_array(V.ActualState).reshape(2, -1).copy()
        uacc0 = ps.get_array(V.UnitAccessories).reshape(64, -1).copy()
        iuacc0 = ps.get_array(V.IntegerUnitAccessories).reshape(1, -1).copy()
        ps.set_period_analysis(n_an - 1, tol, 0)        # one period more than stored sections
        ps.solve_periods(n_an, -1)
        for v in (V.PoincareSections, V.PeriodNumber, V.MaximumAccessory, V.ActualState):
            ps.SynchroniseFromDeviceToHost(v)
        ps.InsertSynchronisationPoint()
        ps.SynchroniseSolver()
        sec = ps.get_array(V.PoincareSections).reshape(n_an - 1, -1)
        per = ps.get_array(V.PeriodNumber)
        mx = ps.get_array(V.MaximumAccessory)
        st = ps.get_array(V.ActualState).reshape(2, -1)
    finally:
        ps.close()
    w_sec, w_per, w_mx, w_st = _oracle_analysis(oracle_lib, ens, state0, uacc0, iuacc0, n_an, tol, 0)
    assert np.array_equal(st.view(np.int64), w_st.view(np.int64))
    assert np.array_equal(sec.view(np.int64), w_sec[:n_an - 1].view(np.int64))
    assert np.array_equal(per, w_per)
    assert np.array_equal(mx.view(np.int64), w_mx.view(np.int64))


def _fmt(v, width, prec):
    return f"{v:>{width}.{prec}e}"


def test_output_files_have_the_reference_layout(gpu, tmp_path):
    ens = _ensemble()
    ps = ens.make_solver()
    try:
        ps.SynchroniseFromHostToDevice(V.All)
        ps.set_period_analysis(2, 1e-6, 0)
        ps.solve_periods(2, -1)
        ps.SynchroniseFromDeviceToHost(V.All)
        for v in (V.PoincareSections, V.PeriodNumber, V.MaximumAccessory):
            ps.SynchroniseFromDeviceToHost(v)
        ps.InsertSynchronisationPoint()
        ps.SynchroniseSolver()
        for kind in S.CsvKind:
            ps.write_csv(kind, tmp_path / f"{kind.name}.csv")
        up = ps.get_array(V.UnitParameters).reshape(21, -1)
        ua = ps.get_array(V.UnitAccessories).reshape(64, -1)
        sec = ps.get_array(V.PoincareSections).reshape(2, -1)
        per = ps.get_array(V.PeriodNumber)
        mx = ps.get_array(V.MaximumAccessory)
    finally:
        ps.close()
    ns, n = ens.n_systems, 32
    # CollapseStrength.cu:174-198
    lines = (tmp_path / "Collapse.csv").read_text().splitlines()
    assert len(lines) == ns * 32
    s, c = 3, 5
    want = (f"{s:>6}," + _fmt(up[15, s * n], 17, 10) + "," + _fmt(up[16, s * n], 17, 10) + ","
            + "".join(_fmt(ua[c, s * n + u], 10, 3) + "," for u in range(n))
            + "".join(_fmt(ua[c + 32, s * n + u], 10, 3) + "," for u in range(n)))
    assert lines[s * 32 + c] == want
    # BubbleEnsemble.cu:435-455, two sections appended
    lines = (tmp_path / "Poincare.csv").read_text().splitlines()
    assert len(lines) == 2 * ns
    k, s = 1, 2
    want = f"{s:>4}," + _fmt(up[15, s * n], 18, 10) + "," + "".join(_fmt(sec[k, s * n + u], 18, 10) + "," for u in range(n))
    assert lines[k * ns + s] == want
    # BubbleEnsemble.cu:457-491
    lines = (tmp_path / "Period.csv").read_text().splitlines()
    assert lines[s] == f"{s:>4}," + _fmt(up[15, s * n], 18, 10) + "," + "".join(f"{per[s * n + u]:>4}," for u in range(n))
    lines = (tmp_path / "Expansion.csv").read_text().splitlines()
    assert lines[s] == f"{s:>4}," + _fmt(up[16, s * n], 18, 10) + "," + "".join(f"{int(mx[s * n + u]):>4}," for u in range(n))


def test_print_files_have_the_reference_layout(gpu, tmp_path):
    """Print(var) / Print(var, n) (Interface.cuh:1809-1947): width 18, 10 digits,
    a comma after every value; dense output with its header blocks."""
    ens = W.c1_ensemble().subset([3, 40])
    ens.max_steps_per_period = 50_000
    ps = ens.make_solver(n_dense_output=4)
    try:
        ps.SolverOption(S.ListOfSolverOptions.DenseOutputMinimumTimeStep, 0.2)
        ps.SynchroniseFromHostToDevice(V.All)
        ps.solve_periods(1, -1)
        ps.SynchroniseFromDeviceToHost(V.All)
        ps.InsertSynchronisationPoint()
        ps.SynchroniseSolver()
        for v in (V.ActualState, V.TimeDomain, V.IntegerUnitAccessories):
            ps.Print(v, directory=tmp_path)
        ps.Print(V.CouplingMatrix, 0, directory=tmp_path)
        ps.Print(V.DenseOutput, 1, directory=tmp_path)
        st = ps.get_array(V.ActualState).reshape(2, -1)
        td = ps.get_array(V.TimeDomain).reshape(2, -1)
        iu = ps.get_array(V.IntegerUnitAccessories)
        C = ps.get_array(V.CouplingMatrix)
        dt = ps.get_array(V.DenseTime).reshape(4, -1)
        ds = ps.get_array(V.DenseState).reshape(4, 2, -1)
        di = ps.get_array(V.DenseIndex)
        up = ps.get_array(V.UnitParameters).reshape(21, -1)
    finally:
        ps.close()
    f18 = lambda v: f"{v:>18.10e}"
    lines = (tmp_path / "ActualStateInSolverObject.txt").read_text().splitlines()
    assert len(lines) == 64 and lines[37] == f18(st[0, 37]) + "," + f18(st[1, 37]) + ","
    lines = (tmp_path / "TimeDomainInSolverObject.txt").read_text().splitlines()
    assert lines[1] == f18(td[0, 1]) + "," + f18(td[1, 1]) + ","
    lines = (tmp_path / "IntegerUnitAccessoriesInSolverObject.txt").read_text().splitlines()
    assert lines[5] == f"{iu[5]:>18}" + ","
    lines = (tmp_path / "CouplingMatrixInSolverObject_0.txt").read_text().splitlines()
    assert lines[2] == "".join(f18(C[2 + 32 * j]) + "," for j in range(32))
    text = (tmp_path / "DenseOutput_1.txt").read_text().split("\n")
    assert text[0] == "UnitParameters:"
    assert text[1] == f"{'Serial No.':>18}," + ",".join(f"{'U' + str(u):>18}" for u in range(32))
    assert text[2] == f"{0:>18}," + ",".join(f18(up[0, 32 + u]) for u in range(32))
    k = text.index("Time series:")
    rows = text[k + 2:k + 2 + int(di[1])]
    assert len(rows) == int(di[1]) >= 1
    assert rows[0] == f18(dt[0, 1]) + "," + ",".join(f18(ds[0, c, 32 + u]) for u in range(32) for c in range(2))
