/*
 * km_model.cuh -- the default system definition compiled into the solver:
 * coupled Keller-Miksis bubbles with collapse bookkeeping.
 *
 * The seven callbacks keep the names and argument lists of the reference's
 * user interface (BubbleEnsemble_SystemDefinition.cuh:8, :52, :69, :79, :97,
 * :108, :119), so a user's own system-definition header can replace this one
 * at build time (BES_SYSTEM_DEFINITION).  The arithmetic restates
 * BubbleEnsemble_SystemDefinition.cuh:15-45 with explicit fused multiply-adds
 * and the project's own elementary functions (bes_math.cuh).
 *
 * A system definition also declares its sizes through the BES_MODEL_*
 * macros below; they correspond to the reference's template parameters
 * UD, NUP, NSP, NGP, NiGP, NUA, NiUA, NSA, NiSA and NE
 * (CollapseStrength.cu:36-53).
 */
#ifndef BES_KM_MODEL_CUH
#define BES_KM_MODEL_CUH

#include "bes_math.cuh"

#ifndef NCOLL
#define NCOLL 32             /* recorded collapses per unit (CollapseStrength.cu:22) */
#endif

#define BES_MODEL_NAME "keller_miksis_collapse"
#define BES_MODEL_UD 2       /* R/R_E, dR/dtau */
#define BES_MODEL_NUP 21     /* CollapseStrength.cu:337-357 */
#define BES_MODEL_NSP 0
#define BES_MODEL_NGP 0
#define BES_MODEL_NIGP 0
#define BES_MODEL_NUA (2 * NCOLL)
#define BES_MODEL_NIUA 1
#define BES_MODEL_NSA 0
#define BES_MODEL_NISA 0
#define BES_MODEL_NE 1
/* the coupled acceleration is component 1; component 0 enters the operator as X0^2 */
#define BES_MODEL_IMPLICIT_COMPONENT 1

#define BES_KM_PI 3.14159265358979323846

/* Right-hand side, BubbleEnsemble_SystemDefinition.cuh:8-49.
 * F[0] = X1, F[1] = N/D (uncoupled acceleration), CPT = -2 X0 X1^2, CPF = 1/D. */
template <class Precision>
__forceinline__ __device__ void CoupledSystems_PerBlock_OdeFunction(
    int sid, int uid,
    Precision* F, Precision* X, Precision T,
    Precision* uPAR, Precision* sPAR, Precision* gPAR, int* igPAR,
    Precision* uACC, int* iuACC, Precision* sACC, int* isACC,
    Precision* CPT, Precision* CPF)
{
    Precision rx1 = 1.0 / X[0];
    Precision p = bes::math::pow_recip(X[0], uPAR[10]);   /* (1/X0)^(3 kappa), off the reciprocal's chain */
    Precision s1, c1;
    bes::math::sincospi(2.0 * T, s1, c1);
    Precision s2, c2;
    if (uPAR[11] == 0.0 && uPAR[12] == 0.0) {
        s2 = 0.0; c2 = 1.0;
    } else {
        bes::math::sincos(fma(2.0 * uPAR[11] * BES_KM_PI, T, uPAR[12]), s2, c2);
    }
    Precision g = fma(uPAR[9], X[1], 1.0);
    Precision N = fma(uPAR[1], X[1], uPAR[0]) * p;
    N = fma(-uPAR[2], g, N);
    N = fma(-uPAR[3], rx1, N);
    N = fma(-(uPAR[4] * X[1]), rx1, N);
    Precision h = fma(-0.5 * uPAR[9], X[1], 1.5);
    N = fma(-(h * X[1]), X[1], N);
    Precision sd = fma(uPAR[6], s2, uPAR[5] * s1);
    N = fma(-sd, g, N);
    Precision cd = fma(uPAR[8], c2, uPAR[7] * c1);
    N = fma(-X[0], cd, N);
    Precision D = fma(uPAR[4], uPAR[9], fma(-(uPAR[9] * X[0]), X[1], X[0]));
    Precision rD = 1.0 / D;
    F[0] = X[1];
    F[1] = N * rD;
    CPT[0] = (-2.0 * X[0] * X[1]) * X[1];
    CPF[0] = rD;
}

/* Never called by the reference solver either (BubbleEnsemble_SystemDefinition.cuh:52-64). */
template <class Precision>
__forceinline__ __device__ void CoupledSystems_PerBlock_UpdateCouplingTerm(
    int sid, int uid,
    Precision* F, Precision* X, Precision T,
    Precision* uPAR, Precision* sPAR, Precision* gPAR, int* igPAR,
    Precision* uACC, int* iuACC, Precision* sACC, int* isACC,
    Precision* CPT, Precision* CPF)
{
    CPT[0] = -(2 * X[0] * X[1] * X[1] + X[0] * X[0] * F[1]);
}

/* Event: radius extremum, dR/dtau = 0 (BubbleEnsemble_SystemDefinition.cuh:69-76). */
template <class Precision>
__forceinline__ __device__ void CoupledSystems_PerBlock_EventFunction(
    int sid, int uid, Precision* EF,
    Precision T, Precision dT, Precision* TD, Precision* X,
    Precision* uPAR, Precision* sPAR, Precision* gPAR, int* igPAR,
    Precision* uACC, int* iuACC, Precision* sACC, int* isACC)
{
    EF[0] = X[1];
}

/* Radius maximum found: store it and start tracking the following minimum
 * (BubbleEnsemble_SystemDefinition.cuh:79-92). */
template <class Precision>
__forceinline__ __device__ void CoupledSystems_PerBlock_ActionAfterEventDetection(
    int sid, int uid, int IDX, int& UDT,
    Precision& T, Precision& dT, Precision* TD, Precision* X,
    Precision* uPAR, Precision* sPAR, Precision* gPAR, int* igPAR,
    Precision* uACC, int* iuACC, Precision* sACC, int* isACC)
{
    iuACC[0]++;
    if (iuACC[0] < NCOLL) {
        uACC[iuACC[0]] = X[0];
        uACC[iuACC[0] + NCOLL] = X[0];
    }
}

/* Track the radius minimum after the last maximum at accepted step ends
 * (BubbleEnsemble_SystemDefinition.cuh:97-105). */
template <class Precision>
__forceinline__ __device__ void CoupledSystems_PerBlock_ActionAfterSuccessfulTimeStep(
    int sid, int uid, int& UDT,
    Precision& T, Precision& dT, Precision* TD, Precision* X,
    Precision* uPAR, Precision* sPAR, Precision* gPAR, int* igPAR,
    Precision* uACC, int* iuACC, Precision* sACC, int* isACC)
{
    if ((iuACC[0] < NCOLL) && (X[0] < uACC[iuACC[0] + NCOLL]))
        uACC[iuACC[0] + NCOLL] = X[0];
}

/* Each period starts at TD[0] (BubbleEnsemble_SystemDefinition.cuh:108-116). */
template <class Precision>
__forceinline__ __device__ void CoupledSystems_PerBlock_Initialization(
    int sid, int uid, int& DOIDX,
    Precision& T, Precision& dT, Precision* TD, Precision* X,
    Precision* uPAR, Precision* sPAR, Precision* gPAR, int* igPAR,
    Precision* uACC, int* iuACC, Precision* sACC, int* isACC)
{
    if (uid == 0) T = TD[0];
}

template <class Precision>
__forceinline__ __device__ void CoupledSystems_PerBlock_Finalization(
    int sid, int uid, int& DOIDX,
    Precision& T, Precision& dT, Precision* TD, Precision* X,
    Precision* uPAR, Precision* sPAR, Precision* gPAR, int* igPAR,
    Precision* uACC, int* iuACC, Precision* sACC, int* isACC)
{
}

#endif
