"""The C-ABI library loads and exports every entry point include/bes.h declares.

No compute call is made: the tests use only entry points that need no GPU."""
import ctypes
import re
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]


def declared_symbols():
    text = (ROOT / "include" / "bes.h").read_text()
    return sorted(set(re.findall(r"^\s*(?:bes_status|const char\*)\s+(bes_\w+)\s*\(", text, re.M)))


def test_header_declares_entry_points():
    syms = declared_symbols()
    assert len(syms) >= 35
    assert "bes_create" in syms and "bes_solve_periods" in syms


def test_library_exports_every_declared_symbol(bes_lib):
    from bubbleensemble_implicitextension_b200 import solver
    for name in declared_symbols():
        assert hasattr(bes_lib, name), name
        assert name in solver.SIGNATURES, f"{name} lacks a ctypes signature"


def test_model_info(bes_lib):
    from bubbleensemble_implicitextension_b200 import solver
    info = solver.model_info()
    assert info.name == b"keller_miksis_collapse"
    assert (info.unit_dim, info.n_unit_parameters, info.n_unit_accessories, info.n_int_unit_accessories,
            info.n_events) == (2, 21, 64, 1, 1)


def test_status_strings(bes_lib):
    assert bes_lib.bes_status_string(0) == b"ok"
    assert bes_lib.bes_status_string(2) == b"index out of range"


def test_text_loaders(tmp_path, bes_lib):
    from bubbleensemble_implicitextension_b200 import solver
    r = np.array([7.8364451240181, 3.1521700965666, 2.8332452169749])
    (tmp_path / "sizes.txt").write_text("\n".join(f"{x:+.13e}" for x in r) + "\n")
    np.testing.assert_array_equal(solver.load_bubble_sizes(tmp_path / "sizes.txt", 3), r)
    rows = [[f"{v:+.13e}" for v in row] for row in np.arange(9, dtype=float).reshape(3, 3) * 1e-4]
    M = np.array([[float(v) for v in row] for row in rows])
    (tmp_path / "c.txt").write_text("\n".join(" ".join(row) for row in rows) + "\n")
    np.testing.assert_array_equal(solver.load_coupling_matrix(tmp_path / "c.txt", 3), M)
    with pytest.raises(solver.BesError) as e:
        solver.load_bubble_sizes(tmp_path / "sizes.txt", 4)
    assert e.value.status == 6
    with pytest.raises(solver.BesError):
        solver.load_bubble_sizes(tmp_path / "missing.txt", 1)


def test_create_validates_sizes_before_touching_a_device(bes_lib):
    from bubbleensemble_implicitextension_b200 import solver
    info = solver.ModelInfo()
    bes_lib.bes_model_info_get(ctypes.byref(info))
    info.n_unit_parameters = 20
    with pytest.raises(solver.BesError) as e:
        solver.ProblemSolver(4, 32, model=info)
    assert e.value.status == 7
