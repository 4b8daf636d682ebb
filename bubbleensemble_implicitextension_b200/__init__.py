"""B200-native ensemble integrator for coupled Keller-Miksis bubble systems.

The compute path is ``libbes.so`` (hand-written sm_100a CUDA behind the C ABI
of ``include/bes.h``); :mod:`.solver` binds it with the names of the
reference's ``ProblemSolver`` and :mod:`.workloads` builds ensembles.
"""
from . import solver, workloads  # noqa: F401
from .solver import BesError, ProblemSolver, load_library  # noqa: F401

__all__ = ["solver", "workloads", "BesError", "ProblemSolver", "load_library"]
