/* Drop-in replacement of the reference's SourceCodes/CoupledSystems_PerBlock_Interface.cuh:
 * put this directory first on the include path of a reference driver and link
 * libbes.so; the driver's ProblemSolver<...> then runs on the B200 library. */
#ifndef BES_DROPIN_INTERFACE_CUH
#define BES_DROPIN_INTERFACE_CUH
#include "../bes_problem_solver.h"
#endif
