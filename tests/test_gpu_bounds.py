"""The reference's run-time checks (BoundCheck on every SetHost / GetHost /
SolverOption index, Interface.cuh:718-733) as status codes: out-of-range
system, unit, component and matrix indices, a variable given to the wrong
overload and an invalid option value are refused without touching the data."""
import numpy as np
import pytest

from bubbleensemble_implicitextension_b200 import solver as S
from bubbleensemble_implicitextension_b200 import workloads as W

pytestmark = pytest.mark.gpu
V = S.ListOfVariables
O = S.ListOfSolverOptions
ERR_INDEX, ERR_OPTION, ERR_ARGUMENT = 2, 3, 1


def test_index_and_option_checks(gpu):
    ens = W.c1_ensemble(n_pa=2, n_f=1)
    ps = ens.make_solver()
    try:
        before = ps.get_array(V.ActualState).copy()
        for args in [(2, 0, V.ActualState, 0, 1.0),      # system 2 of 2
                     (0, 32, V.ActualState, 0, 1.0),     # unit 32 of 32
                     (0, 0, V.ActualState, 2, 1.0),      # component 2 of UD = 2
                     (0, 0, V.UnitParameters, 21, 1.0)]:
            with pytest.raises(S.BesError, match="out of range") as e:
                ps.SetHost(*args)
            assert e.value.status == ERR_INDEX
        with pytest.raises(S.BesError) as e:
            ps.SetHost(0, V.CouplingMatrix, 32, 0, 1.0)   # row 32 of a 32 x 32 matrix
        assert e.value.status == ERR_INDEX
        with pytest.raises(S.BesError) as e:
            ps.GetHost(1, V.CouplingMatrix, 0, 0)         # one matrix only
        assert e.value.status == ERR_INDEX
        with pytest.raises(S.BesError, match="different argument list") as e:
            ps.SetHost(0, 0, V.TimeDomain, 0, 1.0)        # system-scope variable in the unit overload
        assert e.value.status == ERR_OPTION
        with pytest.raises(S.BesError) as e:
            ps.SolverOption(O.MaxStepsPerPeriod, 0)
        assert e.value.status == ERR_ARGUMENT
        assert np.array_equal(ps.get_array(V.ActualState), before)
    finally:
        ps.close()
