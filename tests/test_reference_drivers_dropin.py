"""The reference's own driver programs (CollapseStrength.cu, BubbleEnsemble.cu)
compile unchanged against include/dropin/ and link with libbes.so: the
drivers' ProblemSolver<NS,UPS,...> (SourceCodes/CoupledSystems_PerBlock_Interface.cuh:
135-248, used at CollapseStrength.cu:84-151 and BubbleEnsemble.cu:95-168) is
the library's C++ shim.  Compiling is the check; the drivers' own sweeps
(101 x 101 points x 512 periods) are not run.  Skipped where the reference
tree is not available (the GPU machines)."""
import subprocess

import pytest

from oracle import build_ref


def test_reference_drivers_build_against_dropin(tmp_path, bes_lib):
    if build_ref.reference_dir() is None or not (build_ref.reference_dir() / "CollapseStrength.cu").exists():
        pytest.skip("reference tree not available")
    exes = build_ref.build_reference_drivers(tmp_path)
    assert set(exes) == {"CollapseStrength", "BubbleEnsemble"}
    for drv, exe in exes.items():
        assert exe.exists()
        dyn = subprocess.run(["readelf", "-d", str(exe)], capture_output=True, text=True).stdout
        assert "libbes.so" in dyn, f"{drv} is not linked against libbes.so"
        syms = subprocess.run(["nm", "-D", "--undefined-only", str(exe)], capture_output=True, text=True).stdout
        assert "bes_create" in syms and "bes_solve" in syms, f"{drv} does not call the C ABI"
