/*
 * bes_problem_solver.h -- header-only drop-in for the reference's host API.
 *
 * Rebuilds the class template
 *   ProblemSolver<NS,UPS,UD,TPB,SPB,NC,CBW,CCI,NUP,NSP,NGP,NiGP,NUA,NiUA,NSA,NiSA,NE,NDO,Algorithm,Precision>
 * of SourceCodes/CoupledSystems_PerBlock_Interface.cuh:135-248 on top of the
 * C ABI in bes.h, with the same enumerations (ListOfVariables,
 * ListOfSolverOptions, Algorithms; Interface.cuh:33-68), member names,
 * overloads and argument meaning, so a driver written for the reference
 * (e.g. CollapseStrength.cu:84-151) compiles against it by swapping the
 * include.  Like the reference, a failed call prints the reason and calls
 * exit(EXIT_FAILURE) (Interface.cuh:13-22, :718-733).
 *
 * Differences: Precision must be double (the library integrates in FP64);
 * TPB and SPB are accepted and ignored (the library picks its own launch
 * shape: one warp per system); the device callbacks are the ones compiled
 * into libbes.so (BES_SYSTEM_DEFINITION at build time), so the driver does
 * not include a system-definition header.  Solve() launches one period
 * asynchronously, as the reference does; SolvePeriods(n, reset_at) is the
 * persistent multi-period extension.
 *
 * Plain C++: needs bes.h and libbes.so, not the CUDA headers.
 */
#ifndef BES_PROBLEM_SOLVER_H
#define BES_PROBLEM_SOLVER_H

#include <cstdlib>
#include <fstream>
#include <iomanip>
#include <iostream>
#include <string>
#include <type_traits>
#include <vector>

#include "bes.h"

enum Algorithms { RK4 = BES_RK4, RKCK45 = BES_RKCK45 };

enum ListOfVariables {
    All = BES_ALL, TimeDomain = BES_TIME_DOMAIN, ActualTime = BES_ACTUAL_TIME, ActualState = BES_ACTUAL_STATE,
    UnitParameters = BES_UNIT_PARAMETERS, SystemParameters = BES_SYSTEM_PARAMETERS,
    GlobalParameters = BES_GLOBAL_PARAMETERS, IntegerGlobalParameters = BES_INTEGER_GLOBAL_PARAMETERS,
    UnitAccessories = BES_UNIT_ACCESSORIES, IntegerUnitAccessories = BES_INTEGER_UNIT_ACCESSORIES,
    SystemAccessories = BES_SYSTEM_ACCESSORIES, IntegerSystemAccessories = BES_INTEGER_SYSTEM_ACCESSORIES,
    CouplingMatrix = BES_COUPLING_MATRIX, CouplingStrength = BES_COUPLING_STRENGTH,
    CouplingIndex = BES_COUPLING_INDEX, DenseOutput = BES_DENSE_OUTPUT, DenseIndex = BES_DENSE_INDEX,
    DenseTime = BES_DENSE_TIME, DenseState = BES_DENSE_STATE
};

enum ListOfSolverOptions {
    InitialTimeStep = BES_OPT_INITIAL_TIME_STEP, ActiveSystems = BES_OPT_ACTIVE_SYSTEMS,
    MaximumTimeStep = BES_OPT_MAXIMUM_TIME_STEP, MinimumTimeStep = BES_OPT_MINIMUM_TIME_STEP,
    TimeStepGrowLimit = BES_OPT_TIME_STEP_GROW_LIMIT, TimeStepShrinkLimit = BES_OPT_TIME_STEP_SHRINK_LIMIT,
    RelativeTolerance = BES_OPT_RELATIVE_TOLERANCE, AbsoluteTolerance = BES_OPT_ABSOLUTE_TOLERANCE,
    EventTolerance = BES_OPT_EVENT_TOLERANCE, EventDirection = BES_OPT_EVENT_DIRECTION,
    DenseOutputSaveFrequency = BES_OPT_DENSE_OUTPUT_SAVE_FREQUENCY,
    DenseOutputMinimumTimeStep = BES_OPT_DENSE_OUTPUT_MINIMUM_TIME_STEP,
    SharedGlobalVariables = BES_OPT_SHARED_GLOBAL_VARIABLES, SharedCouplingMatrices = BES_OPT_SHARED_COUPLING_MATRICES
};

namespace bes_shim {
inline void check(bes_status s, const bes_solver* h, const char* where) {
    if (s != BES_OK) {
        std::cerr << "ERROR: In solver member function " << where << "!" << std::endl;
        std::cerr << "       " << bes_status_string(s) << ": " << bes_last_error(h) << std::endl;
        std::exit(EXIT_FAILURE);
    }
}
}  // namespace bes_shim

/* ListCUDADevices, Interface.cuh:260-296 */
inline void ListCUDADevices() {
    int32_t n = 0;
    bes_device_count(&n);
    std::cout << "Number of CUDA devices: " << n << std::endl;
    for (int d = 0; d < n; d++) {
        bes_device_info info;
        if (bes_device_info_get(d, &info) == BES_OK)
            std::cout << "  device " << d << ": " << info.name << ", compute capability " << info.cc_major << "."
                      << info.cc_minor << std::endl;
    }
}

/* SelectDeviceByClosestRevision, Interface.cuh:298-312 */
inline int SelectDeviceByClosestRevision(int MajorRevision, int MinorRevision) {
    int32_t n = 0;
    bes_device_count(&n);
    int best = 0, best_gap = 1 << 30;
    for (int d = 0; d < n; d++) {
        bes_device_info info;
        if (bes_device_info_get(d, &info) != BES_OK) continue;
        int gap = std::abs((info.cc_major * 10 + info.cc_minor) - (MajorRevision * 10 + MinorRevision));
        if (gap < best_gap) { best_gap = gap; best = d; }
    }
    return best;
}

/* PrintPropertiesOfSpecificDevice, Interface.cuh:314-346 */
inline void PrintPropertiesOfSpecificDevice(int SelectedDevice) {
    bes_device_info info;
    if (bes_device_info_get(SelectedDevice, &info) != BES_OK) {
        std::cout << "Device " << SelectedDevice << " is not available" << std::endl;
        return;
    }
    std::cout << "Device " << SelectedDevice << ": " << info.name << std::endl;
    std::cout << "   Compute capability: " << info.cc_major << "." << info.cc_minor << std::endl;
    std::cout << "   Multiprocessors:    " << info.multiprocessors << std::endl;
    std::cout << "   Global memory:      " << info.global_memory_bytes / (1024 * 1024) << " Mb" << std::endl;
}

template <int NS, int UPS, int UD, int TPB, int SPB, int NC, int CBW, int CCI, int NUP, int NSP, int NGP, int NiGP,
          int NUA, int NiUA, int NSA, int NiSA, int NE, int NDO, Algorithms Algorithm, class Precision>
class ProblemSolver {
    static_assert(std::is_same<Precision, double>::value, "the B200 solver integrates in FP64 (Precision = double)");

  public:
    explicit ProblemSolver(int Device) {
        bes_config c = {};
        c.device = Device;
        c.n_systems = NS;
        c.units_per_system = UPS;
        c.unit_dim = UD;
        c.n_unit_parameters = NUP;
        c.n_system_parameters = NSP;
        c.n_global_parameters = NGP;
        c.n_int_global_parameters = NiGP;
        c.n_unit_accessories = NUA;
        c.n_int_unit_accessories = NiUA;
        c.n_system_accessories = NSA;
        c.n_int_system_accessories = NiSA;
        c.n_events = NE;
        c.n_dense_output = NDO;
        c.n_couplings = NC;
        c.coupling_bandwidth = CBW;
        c.coupling_circular = CCI;
        c.algorithm = Algorithm;
        c.n_coupling_matrices = 1;
        bes_shim::check(bes_create(&c, &h_), nullptr, "ProblemSolver");
    }
    ~ProblemSolver() {
        if (h_) bes_destroy(h_);
    }
    ProblemSolver(const ProblemSolver&) = delete;
    ProblemSolver& operator=(const ProblemSolver&) = delete;

    template <typename T> void SolverOption(ListOfSolverOptions Option, T Value) {
        bes_shim::check(bes_solver_option(h_, Option, (double)Value), h_, "SolverOption");
    }
    template <typename T> void SolverOption(ListOfSolverOptions Option, int Index, T Value) {
        bes_shim::check(bes_solver_option_indexed(h_, Option, Index, (double)Value), h_, "SolverOption");
    }

    /* unit scope */
    template <typename T> void SetHost(int SystemNumber, int UnitNumber, ListOfVariables Variable, int SerialNumber, T Value) {
        bes_shim::check(bes_set_host_unit(h_, SystemNumber, UnitNumber, Variable, SerialNumber, (double)Value), h_, "SetHost");
    }
    /* system scope and dense time */
    template <typename T> void SetHost(int SystemNumber, ListOfVariables Variable, int SerialNumber, T Value) {
        bes_shim::check(bes_set_host_system(h_, SystemNumber, Variable, SerialNumber, (double)Value), h_, "SetHost");
    }
    /* global scope */
    template <typename T> void SetHost(ListOfVariables Variable, int SerialNumber, T Value) {
        bes_shim::check(bes_set_host_global(h_, Variable, SerialNumber, (double)Value), h_, "SetHost");
    }
    /* coupling matrix */
    template <typename T> void SetHost(int CouplingNumber, ListOfVariables Variable, int Row, int Col, T Value) {
        bes_shim::check(bes_set_host_coupling(h_, CouplingNumber, Variable, Row, Col, (double)Value), h_, "SetHost");
    }
    /* dense index */
    template <typename T> void SetHost(int SystemNumber, ListOfVariables Variable, T Value) {
        bes_shim::check(bes_set_host_dense_index(h_, SystemNumber, Variable, (double)Value), h_, "SetHost");
    }
    /* dense state */
    template <typename T>
    void SetHost(int SystemNumber, int UnitNumber, ListOfVariables Variable, int ComponentNumber, int SerialNumber, T Value) {
        bes_shim::check(bes_set_host_dense_state(h_, SystemNumber, UnitNumber, Variable, ComponentNumber, SerialNumber,
                                                 (double)Value), h_, "SetHost");
    }

    void SynchroniseFromHostToDevice(ListOfVariables Variable) {
        bes_shim::check(bes_synchronise_host_to_device(h_, Variable), h_, "SynchroniseFromHostToDevice");
    }
    void SynchroniseFromDeviceToHost(ListOfVariables Variable) {
        bes_shim::check(bes_synchronise_device_to_host(h_, Variable), h_, "SynchroniseFromDeviceToHost");
    }

    template <typename T> T GetHost(int SystemNumber, int UnitNumber, ListOfVariables Variable, int SerialNumber) {
        double v;
        bes_shim::check(bes_get_host_unit(h_, SystemNumber, UnitNumber, Variable, SerialNumber, &v), h_, "GetHost");
        return (T)v;
    }
    template <typename T> T GetHost(int SystemNumber, ListOfVariables Variable, int SerialNumber) {
        double v;
        bes_shim::check(bes_get_host_system(h_, SystemNumber, Variable, SerialNumber, &v), h_, "GetHost");
        return (T)v;
    }
    template <typename T> T GetHost(ListOfVariables Variable, int SerialNumber) {
        double v;
        bes_shim::check(bes_get_host_global(h_, Variable, SerialNumber, &v), h_, "GetHost");
        return (T)v;
    }
    template <typename T> T GetHost(int CouplingNumber, ListOfVariables Variable, int Row, int Col) {
        double v;
        bes_shim::check(bes_get_host_coupling(h_, CouplingNumber, Variable, Row, Col, &v), h_, "GetHost");
        return (T)v;
    }
    template <typename T> T GetHost(int SystemNumber, ListOfVariables Variable) {
        double v;
        bes_shim::check(bes_get_host_dense_index(h_, SystemNumber, Variable, &v), h_, "GetHost");
        return (T)v;
    }
    template <typename T>
    T GetHost(int SystemNumber, int UnitNumber, ListOfVariables Variable, int ComponentNumber, int SerialNumber) {
        double v;
        bes_shim::check(bes_get_host_dense_state(h_, SystemNumber, UnitNumber, Variable, ComponentNumber, SerialNumber, &v),
                        h_, "GetHost");
        return (T)v;
    }

    /* Print(ListOfVariables) and Print(ListOfVariables, int), Interface.cuh:1809-1947:
     * the host mirror to <Variable>InSolverObject.txt (DenseOutput_<n>.txt,
     * CouplingMatrixInSolverObject_<n>.txt) in the reference's format */
    void Print(ListOfVariables Variable) { bes_shim::check(bes_print(h_, Variable, 0, nullptr), h_, "Print"); }
    void Print(ListOfVariables Variable, int SerialNumber) {
        bes_shim::check(bes_print(h_, Variable, SerialNumber, nullptr), h_, "Print");
    }

    void Solve() { bes_shim::check(bes_solve(h_), h_, "Solve"); }
    /* extension: n_periods Solve() calls (accessories reset before period reset_at) in one launch */
    void SolvePeriods(int n_periods, int reset_at) { bes_shim::check(bes_solve_periods(h_, n_periods, reset_at), h_, "SolvePeriods"); }
    /* extensions: per-period analysis on the device, the drivers' output files, launch-shape autotuning */
    void SetPeriodAnalysis(int sections, double distance_tolerance = 1e-6, int accessory_index = 0) {
        bes_shim::check(bes_set_period_analysis(h_, sections, distance_tolerance, accessory_index), h_,
                        "SetPeriodAnalysis");
    }
    void WriteCSV(int kind, const std::string& path) {
        bes_shim::check(bes_write_csv(h_, kind, path.c_str()), h_, "WriteCSV");
    }
    bes_autotune_result Autotune(int n_periods = 1, int64_t step_cap = 2000) {
        bes_autotune_result r;
        bes_shim::check(bes_autotune(h_, n_periods, step_cap, &r), h_, "Autotune");
        return r;
    }
    void SynchroniseDevice() { bes_shim::check(bes_synchronise_device(h_), h_, "SynchroniseDevice"); }
    void InsertSynchronisationPoint() {
        bes_shim::check(bes_insert_synchronisation_point(h_), h_, "InsertSynchronisationPoint");
    }
    void SynchroniseSolver() { bes_shim::check(bes_synchronise_solver(h_), h_, "SynchroniseSolver"); }

    bes_solver* handle() { return h_; }

  private:
    static const char* VariableName(ListOfVariables v) {
        switch (v) {
            case TimeDomain: return "TimeDomain";
            case ActualTime: return "ActualTime";
            case ActualState: return "ActualState";
            case UnitParameters: return "UnitParameters";
            case SystemParameters: return "SystemParameters";
            case GlobalParameters: return "GlobalParameters";
            case IntegerGlobalParameters: return "IntegerGlobalParameters";
            case UnitAccessories: return "UnitAccessories";
            case IntegerUnitAccessories: return "IntegerUnitAccessories";
            case SystemAccessories: return "SystemAccessories";
            case IntegerSystemAccessories: return "IntegerSystemAccessories";
            case CouplingMatrix: return "CouplingMatrix";
            case CouplingStrength: return "CouplingStrength";
            case CouplingIndex: return "CouplingIndex";
            default: return "Variable";
        }
    }
    bes_solver* h_ = nullptr;
};

#endif
