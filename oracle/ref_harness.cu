/*
 * ref_harness.cu -- TEST INFRASTRUCTURE.  A driver for the reference's own
 * per-block CUDA solver, used to produce golden vectors on the B200 and as
 * the reference arm of the benchmark.  Only the tests, the golden-fixture
 * script and bench.py --impl reference run it.
 *
 * It is compiled (oracle/build_ref.py) against the reference's unmodified
 * headers where they lie: BubbleEnsemble_SystemDefinition.cuh (the user
 * callbacks) and SourceCodes/CoupledSystems_PerBlock_Interface.cuh (the
 * ProblemSolver class and its kernel).  The driving sequence is the one of
 * CollapseStrength.cu:84-151: SolverOption calls, SetHost of every unit
 * parameter / state / accessory and of the coupling matrix,
 * SynchroniseFromHostToDevice(All), one Solve() + InsertSynchronisationPoint()
 * + SynchroniseSolver() per period, the accessory reset before the recorded
 * periods, SynchroniseFromDeviceToHost(All) and GetHost of the results.
 *
 * Compile-time sizes (the reference's template parameters): HARNESS_NS
 * systems of HARNESS_UPS units (TPB = UPS, SPB = 1: the only configuration
 * in which the reference's block reductions are well defined for
 * UPS in {32, 64, 128}), HARNESS_NDO dense-output slots.
 *
 * Input / output are little-endian binary files written / read by
 * oracle/ref_io.py (layout documented there).
 */
#include <chrono>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <vector>

#define NCOLL 32
#include "BubbleEnsemble_SystemDefinition.cuh"
#include "CoupledSystems_PerBlock_Interface.cuh"

#ifndef HARNESS_NS
#define HARNESS_NS 256
#endif
#ifndef HARNESS_UPS
#define HARNESS_UPS 32
#endif
#ifndef HARNESS_NDO
#define HARNESS_NDO 0
#endif

const int NS = HARNESS_NS;
const int UPS = HARNESS_UPS;
const int UD = 2;
const int TPB = UPS;
const int SPB = 1;
const int NC = 1;
const int CBW = 0;
const int CCI = 0;
const int NUP = 21;
const int NSP = 0;
const int NGP = 0;
const int NiGP = 0;
const int NUA = 2 * NCOLL;
const int NiUA = 1;
const int NSA = 0;
const int NiSA = 0;
const int NE = 1;
const int NDO = HARNESS_NDO;

typedef ProblemSolver<NS, UPS, UD, TPB, SPB, NC, CBW, CCI, NUP, NSP, NGP, NiGP, NUA, NiUA, NSA, NiSA, NE, NDO, RKCK45,
                      double>
    Solver;

static const int64_t MAGIC_IN = 0x4245535246494e31LL;   /* "BESRFIN1" */
static const int64_t MAGIC_OUT = 0x42455352464f5531LL;  /* "BESRFOU1" */

static void die(const char* msg) {
    std::fprintf(stderr, "ref_harness: %s\n", msg);
    std::exit(2);
}

template <class T>
static void rd(FILE* f, T* p, size_t n) {
    if (std::fread(p, sizeof(T), n, f) != n) die("short read");
}
template <class T>
static void wr(FILE* f, const T* p, size_t n) {
    if (std::fwrite(p, sizeof(T), n, f) != n) die("short write");
}

int main(int argc, char** argv) {
    if (argc != 3) {
        std::fprintf(stderr, "usage: %s input.bin output.bin\n", argv[0]);
        return 2;
    }
    FILE* fi = std::fopen(argv[1], "rb");
    if (!fi) die("cannot open input");
    int64_t hdr[16];
    rd(fi, hdr, 16);
    if (hdr[0] != MAGIC_IN) die("bad input magic");
    const int ns = (int)hdr[1], ups = (int)hdr[2], ndo = (int)hdr[3], n_periods = (int)hdr[4], reset_at = (int)hdr[5];
    const int evdir = (int)hdr[6], do_freq = (int)hdr[7], device = (int)hdr[8];
    const int restart_each_period = (int)hdr[9]; /* 1: every period starts again from the input state */
    if (ups != UPS) die("unit count differs from the compiled HARNESS_UPS");
    if (ndo != NDO) die("dense-output slots differ from the compiled HARNESS_NDO");
    if (ns < 1 || ns > NS) die("system count outside 1..HARNESS_NS");
    double opt[16];
    rd(fi, opt, 16);
    const double dt0 = opt[0], dtmin = opt[1], dtmax = opt[2], rtol0 = opt[3], rtol1 = opt[4], atol0 = opt[5],
                 atol1 = opt[6], evtol = opt[7], grow = opt[8], shrink = opt[9], do_min_dt = opt[10];
    const int64_t tu = (int64_t)ns * ups;
    std::vector<double> upar(NUP * tu), state(UD * tu), uacc(NUA * tu), coup((size_t)ups * ups);
    std::vector<int32_t> iuacc(tu);
    rd(fi, upar.data(), upar.size());
    rd(fi, state.data(), state.size());
    rd(fi, uacc.data(), uacc.size());
    rd(fi, iuacc.data(), iuacc.size());
    rd(fi, coup.data(), coup.size());
    std::fclose(fi);

    Solver S(device);
    S.SolverOption(SharedCouplingMatrices, 0);
    S.SolverOption(ActiveSystems, ns);
    S.SolverOption(InitialTimeStep, dt0);
    S.SolverOption(MinimumTimeStep, dtmin);
    S.SolverOption(MaximumTimeStep, dtmax);
    S.SolverOption(TimeStepGrowLimit, grow);
    S.SolverOption(TimeStepShrinkLimit, shrink);
    S.SolverOption(RelativeTolerance, 0, rtol0);
    S.SolverOption(RelativeTolerance, 1, rtol1);
    S.SolverOption(AbsoluteTolerance, 0, atol0);
    S.SolverOption(AbsoluteTolerance, 1, atol1);
    S.SolverOption(EventDirection, 0, evdir);
    S.SolverOption(EventTolerance, 0, evtol);
    if (NDO > 0) {
        S.SolverOption(DenseOutputMinimumTimeStep, do_min_dt);
        S.SolverOption(DenseOutputSaveFrequency, do_freq);
    }
    for (int sid = 0; sid < NS; sid++) {
        const int s = sid < ns ? sid : 0; /* inactive systems get a copy of system 0 */
        S.SetHost(sid, TimeDomain, 0, 0.0);
        S.SetHost(sid, TimeDomain, 1, 1.0);
        S.SetHost(sid, ActualTime, 0, 0.0);
        S.SetHost(sid, CouplingStrength, 0, 1.0);
        if (NDO > 0) S.SetHost(sid, DenseIndex, 0);
        for (int uid = 0; uid < UPS; uid++) {
            const int64_t u = (int64_t)s * ups + uid;
            for (int k = 0; k < UD; k++) S.SetHost(sid, uid, ActualState, k, state[k * tu + u]);
            for (int k = 0; k < NUP; k++) S.SetHost(sid, uid, UnitParameters, k, upar[k * tu + u]);
            for (int k = 0; k < NUA; k++) S.SetHost(sid, uid, UnitAccessories, k, uacc[k * tu + u]);
            S.SetHost(sid, uid, IntegerUnitAccessories, 0, iuacc[u]);
        }
    }
    S.SetHost(CouplingIndex, 0, 1);
    for (int r = 0; r < UPS; r++)
        for (int c = 0; c < UPS; c++) S.SetHost(0, CouplingMatrix, r, c, coup[r + (size_t)c * ups]);

    S.SynchroniseFromHostToDevice(All);
    S.InsertSynchronisationPoint();
    S.SynchroniseSolver();
    std::vector<double> period_s(n_periods, 0.0);
    auto t0 = std::chrono::steady_clock::now();
    for (int p = 0; p < n_periods; p++) {
        if (restart_each_period && p > 0) {
            /* the same period again from the input state: SetHost + H2D of the unit-scope state */
            for (int sid = 0; sid < ns; sid++)
                for (int uid = 0; uid < UPS; uid++) {
                    const int64_t u = (int64_t)sid * ups + uid;
                    for (int k = 0; k < UD; k++) S.SetHost(sid, uid, ActualState, k, state[k * tu + u]);
                    for (int k = 0; k < NUA; k++) S.SetHost(sid, uid, UnitAccessories, k, uacc[k * tu + u]);
                    S.SetHost(sid, uid, IntegerUnitAccessories, 0, iuacc[u]);
                }
            S.SynchroniseFromHostToDevice(ActualState);
            S.SynchroniseFromHostToDevice(UnitAccessories);
            S.SynchroniseFromHostToDevice(IntegerUnitAccessories);
            S.InsertSynchronisationPoint();
            S.SynchroniseSolver();
        }
        if (p == reset_at) {
            /* ResetAccessories, CollapseStrength.cu:373-396 */
            for (int sid = 0; sid < NS; sid++)
                for (int uid = 0; uid < UPS; uid++) {
                    for (int k = 0; k < NUA; k++) S.SetHost(sid, uid, UnitAccessories, k, 0.0);
                    S.SetHost(sid, uid, IntegerUnitAccessories, 0, -1);
                }
            S.SynchroniseFromHostToDevice(UnitAccessories);
            S.SynchroniseFromHostToDevice(IntegerUnitAccessories);
        }
        auto tp = std::chrono::steady_clock::now();
        S.Solve();
        S.InsertSynchronisationPoint();
        S.SynchroniseSolver();
        period_s[p] = std::chrono::duration<double>(std::chrono::steady_clock::now() - tp).count();
    }
    auto t1 = std::chrono::steady_clock::now();
    S.SynchroniseFromDeviceToHost(All);
    S.InsertSynchronisationPoint();
    S.SynchroniseSolver();
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        std::fprintf(stderr, "ref_harness: CUDA error %s\n", cudaGetErrorString(e));
        return 3;
    }

    FILE* fo = std::fopen(argv[2], "wb");
    if (!fo) die("cannot open output");
    int64_t oh[8] = {MAGIC_OUT, ns, ups, NDO, (int64_t)std::chrono::duration_cast<std::chrono::nanoseconds>(t1 - t0).count(),
                     n_periods, 0, 0};
    wr(fo, oh, 8);
    std::vector<double> o_state(UD * tu), o_uacc(NUA * tu), o_time(ns), o_dt(NDO > 0 ? NDO * ns : 1),
        o_ds(NDO > 0 ? (size_t)NDO * UD * tu : 1);
    std::vector<int32_t> o_iuacc(tu), o_di(ns);
    for (int sid = 0; sid < ns; sid++) {
        o_time[sid] = S.GetHost<double>(sid, ActualTime, 0);
        o_di[sid] = NDO > 0 ? S.GetHost<int>(sid, DenseIndex) : 0;
        for (int j = 0; j < NDO; j++) o_dt[(size_t)j * ns + sid] = S.GetHost<double>(sid, DenseTime, j);
        for (int uid = 0; uid < UPS; uid++) {
            const int64_t u = (int64_t)sid * ups + uid;
            for (int k = 0; k < UD; k++) o_state[k * tu + u] = S.GetHost<double>(sid, uid, ActualState, k);
            for (int k = 0; k < NUA; k++) o_uacc[k * tu + u] = S.GetHost<double>(sid, uid, UnitAccessories, k);
            o_iuacc[u] = S.GetHost<int>(sid, uid, IntegerUnitAccessories, 0);
            for (int j = 0; j < NDO; j++)
                for (int k = 0; k < UD; k++)
                    o_ds[(size_t)j * UD * tu + k * tu + u] = S.GetHost<double>(sid, uid, DenseState, k, j);
        }
    }
    wr(fo, o_state.data(), o_state.size());
    wr(fo, o_uacc.data(), o_uacc.size());
    wr(fo, o_iuacc.data(), o_iuacc.size());
    wr(fo, o_time.data(), o_time.size());
    wr(fo, o_di.data(), o_di.size());
    if (NDO > 0) {
        wr(fo, o_dt.data(), o_dt.size());
        wr(fo, o_ds.data(), o_ds.size());
    }
    wr(fo, period_s.data(), period_s.size());
    std::fclose(fo);
    std::printf("ref_harness: %d systems x %d units, %d periods, %.6f s\n", ns, ups, n_periods,
                (double)oh[4] * 1e-9);
    return 0;
}
