"""Banded and circular coupling storage (the reference's CBW / CCI modes,
Interface.cuh:1010-1070, ExplicitRungeKutta_Steppers.cuh:586-641): elements set
through SetHost in full-matrix coordinates describe the full matrix of those
formats (the reference's implicit products read full storage in every mode,
Steppers.cuh:660,692).  With CBW > 0 the solve runs the banded operator
(only the 2 CBW + 1 diagonals); with CBW = 1 each row has at most two nonzero
terms, so its sums equal the full matrix's bit for bit, which is what these
tests check (tests/test_gpu_banded.py covers wider bands against the oracle)."""
import numpy as np
import pytest

from bubbleensemble_implicitextension_b200 import solver as S
from bubbleensemble_implicitextension_b200 import workloads as W
from tests.helpers import assert_bitwise

pytestmark = pytest.mark.gpu
V = S.ListOfVariables
KEYS = ["state", "uacc", "iuacc"]


def _ring(n=32, n_sys=3, seed=6):
    """Bubbles on a ring: coupling to the two neighbours only, per-pair factors."""
    rng = np.random.default_rng(seed)
    r = rng.uniform(2.0, 8.0, n)
    C = np.zeros((n, n))
    for i in range(n):
        for j in ((i - 1) % n, (i + 1) % n):
            C[i, j] = r[j] ** 3 / (r[i] ** 2 * 120.0)
    ens = W.c1_ensemble(n_pa=n_sys, n_f=1, n_units=n, n_periods=1, reset_at=-1)
    up = W.km_unit_parameters(ens.info["pa_bar"][:, None], ens.info["f_khz"][:, None], 0.0, 0.0, 0.0, r[None, :])
    ens.upar = up.reshape(W.NUP, -1)
    ens.coupling = C.T.reshape(-1).copy()
    ens.max_steps_per_period = 50_000
    return ens, C


def _solve(ps):
    ps.SynchroniseFromHostToDevice(V.All)
    ps.solve_periods(1, -1)
    ps.SynchroniseFromDeviceToHost(V.All)
    ps.InsertSynchronisationPoint()
    ps.SynchroniseSolver()
    return {"state": ps.get_array(V.ActualState), "uacc": ps.get_array(V.UnitAccessories),
            "iuacc": ps.get_array(V.IntegerUnitAccessories)}


def test_band_storage_equals_full_matrix(gpu):
    ens, C = _ring()
    n = C.shape[0]
    full = ens.make_solver()
    try:
        want = _solve(full)
    finally:
        full.close()
    band = ens.make_solver(coupling_bandwidth=1)
    try:
        band.set_array(V.CouplingMatrix, np.zeros(n * n))
        for i in range(n):
            for j in ((i - 1) % n, (i + 1) % n):
                band.SetHost(0, V.CouplingMatrix, i, j, C[i, j])
        with pytest.raises(S.BesError, match="outside the band"):
            band.SetHost(0, V.CouplingMatrix, 0, 5, 1.0)
        got = _solve(band)
    finally:
        band.close()
    assert_bitwise(got, want, KEYS)


def test_circular_storage_fills_the_circulant(gpu):
    ens, _ = _ring()
    n = 32
    coef = {-1: 0.021, 0: 0.0, 1: 0.034}           # one value per diagonal, every row
    C = np.zeros((n, n))
    for i in range(n):
        for k, c in coef.items():
            C[i, (i + k) % n] = c
    ens.coupling = C.T.reshape(-1).copy()
    full = ens.make_solver()
    try:
        want = _solve(full)
    finally:
        full.close()
    circ = ens.make_solver(coupling_bandwidth=1, coupling_circular=1)
    try:
        circ.set_array(V.CouplingMatrix, np.zeros(n * n))
        for k, c in coef.items():
            circ.SetHost(0, V.CouplingMatrix, 0, k % n, c)   # row 0 sets the diagonal for every row
        assert circ.GetHost(0, V.CouplingMatrix, 17, 18) == coef[1]
        assert circ.GetHost(0, V.CouplingMatrix, 17, 16) == coef[-1]
        got = _solve(circ)
    finally:
        circ.close()
    assert_bitwise(got, want, KEYS)
