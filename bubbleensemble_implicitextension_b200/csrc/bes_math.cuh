/*
 * bes_math.cuh -- double-precision elementary functions used by the solver
 * kernel (pow, exp, log, sinpi/cospi, sin/cos).
 *
 * The reference calls CUDA's device library for these
 * (BubbleEnsemble_SystemDefinition.cuh:16-23,
 * SourceCodes/CoupledSystems_PerBlock_ExplicitRungeKutta_ErrorControllers.cuh:502-505).
 * This file implements them from textbook methods instead, with only +, -,
 * *, /, fma and exponent-field arithmetic, so a host build of the same
 * algorithm gives identical bits:
 *   exp    Cody-Waite reduction by ln 2 (32-bit head + tail), degree-13
 *          Taylor polynomial, exponent-field scaling;
 *   log    x = 2^e m, m in (sqrt2/2, sqrt2], log(1+f) = f - s (f - T(s^2))
 *          with s = f/(2+f) and T the atanh series, kept as head + tail;
 *   pow    exp(y log x) with y*log x carried as head + tail (pow_recip:
 *          (1/x)^y as exp(-y log x));
 *   sinpi  x = n/2 + r, |r| <= 1/4, Taylor series of sin(pi r), cos(pi r);
 *   sin    Cody-Waite reduction by pi/2 in three parts, Taylor series.
 * Coefficients are Taylor coefficients (1/k!, pi^k/k!, 2/(2k+1)) and digit
 * splits of ln 2 and pi/2, rounded to double.  All functions are faithfully
 * rounded (within 1 ulp of the exactly rounded value).
 *
 * The translation unit must be compiled with --fmad=false: every fused
 * multiply-add is written out explicitly.
 */
#ifndef BES_MATH_CUH
#define BES_MATH_CUH

#include <stdint.h>

namespace bes {
namespace math {

__device__ __forceinline__ double round_nearest(double x) {
    const double M = 6755399441055744.0; /* 1.5 * 2^52 */
    if (fabs(x) >= 2251799813685248.0) return x;
    double t = x + M;
    return t - M;
}

__device__ __forceinline__ double pow2_scale(double x, int k) {
    if (k > 1023) {
        x = x * __longlong_as_double((long long)(1023 + 1023) << 52);
        k -= 1023;
        if (k > 1023) return x * __longlong_as_double(0x7ff0000000000000LL);
        return x * __longlong_as_double((long long)(k + 1023) << 52);
    }
    if (k < -1022) {
        x = x * __longlong_as_double((long long)(-1000 + 1023) << 52);
        k += 1000;
        if (k < -1022) return x * 0.0;
        return x * __longlong_as_double((long long)(k + 1023) << 52);
    }
    return x * __longlong_as_double((long long)(k + 1023) << 52);
}

/* ---------------------------------------------------------------------------
 * Division by a divisor known ahead of time.  recip_estimate(b) is the
 * hardware's approximate reciprocal refined by one Newton-Raphson step
 * y <- y + y (1 - b y), with no branches, so it can be computed off the
 * critical path as soon as b is known.  div_markstein(a, b, y, ok) then forms
 * the quotient by Markstein's correction q1 = q0 + (a - b q0) y, q0 = a y
 * (P. Markstein, IBM J. Res. Dev. 34 (1990) 111-119): the Newton step
 * squares the relative error of the hardware estimate and the correction
 * squares that of y again, so q1 is the rounded quotient unless a / b lies
 * very close to a rounding boundary.
 * ok reports the proof that it is: the exact remainder r1 = a - b q1 (one
 * fma) satisfies |r1| < ulp(q1)/2 |b|, with q1 not a power of two (so the ulp
 * is the same on both sides of q1) and a, b within [2^-400, 2^400] (no
 * overflow, underflow or subnormal along the way).  The test is sound for any
 * y: rounding is monotonic and ulp(q1)/2 |b| is exact, so a rounded remainder
 * below the bound means the exact one is.  A caller may go on with q1 before
 * ok is known and redo the work that used it when ok is false, which keeps
 * the test off its dependency chain.  div_known(a, b, y) returns q1 when ok
 * and the IEEE quotient otherwise; both therefore always give the correctly
 * rounded a / b. */
__device__ __forceinline__ double recip_estimate(double b) {
    double y;
    asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(b));
    const double e = fma(-b, y, 1.0);
    return fma(y, e, y);
}

static __device__ __noinline__ double div_ieee(double a, double b) { return a / b; }

__device__ __forceinline__ double div_markstein(double a, double b, double y, bool& ok) {
    const double q0 = a * y;
    const double r0 = fma(-q0, b, a);
    const double q1 = fma(r0, y, q0);
    const double r1 = fma(-q1, b, a);
    const long long qb = __double_as_longlong(q1);
    const double half_ulp_b = __longlong_as_double(qb & 0x7ff0000000000000LL) * 0x1p-53 * fabs(b);
    const double aa = fabs(a), ab = fabs(b);
    ok = aa >= 0x1p-400 && aa <= 0x1p400 && ab >= 0x1p-400 && ab <= 0x1p400 &&
         (qb & 0x000fffffffffffffLL) != 0 && fabs(r1) < half_ulp_b;
    return q1;
}

__device__ __forceinline__ double div_known(double a, double b, double y) {
    bool ok;
    const double q1 = div_markstein(a, b, y, ok);
    if (__builtin_expect(!ok, 0)) return div_ieee(a, b);
    return q1;
}

#define BES_LN2_HI 0.6931471806019545
#define BES_LN2_LO (-4.2009150726810846e-11)
#define BES_INV_LN2 1.4426950408889634
#define BES_SQRT2 1.4142135623730951

/* exp(a + b) with b a small correction */
__device__ __forceinline__ double exp_ab(double a, double b) {
    if (a != a) return a;
    if (a > 709.8) return __longlong_as_double(0x7ff0000000000000LL);
    if (a < -745.2) return 0.0;
    double kd = round_nearest(a * BES_INV_LN2);
    double r = fma(-kd, BES_LN2_HI, a);
    r = fma(-kd, BES_LN2_LO, r);
    r = r + b;
    double p = 1.6059043836821613e-10;
    p = fma(p, r, 2.08767569878681e-09);
    p = fma(p, r, 2.505210838544172e-08);
    p = fma(p, r, 2.755731922398589e-07);
    p = fma(p, r, 2.7557319223985893e-06);
    p = fma(p, r, 2.48015873015873e-05);
    p = fma(p, r, 0.0001984126984126984);
    p = fma(p, r, 0.001388888888888889);
    p = fma(p, r, 0.008333333333333333);
    p = fma(p, r, 0.041666666666666664);
    p = fma(p, r, 0.16666666666666666);
    p = fma(p, r, 0.5);
    p = fma(p, r, 1.0);
    p = fma(p, r, 1.0);
    return pow2_scale(p, (int)kd);
}

/* log(x) as head + tail, x finite and > 0 */
__device__ __forceinline__ void log_hl(double x, double& hi, double& lo) {
    int e = 0;
    if (x < 2.2250738585072014e-308) { x = x * 18014398509481984.0; e = -54; }
    unsigned long long u = (unsigned long long)__double_as_longlong(x);
    e += (int)((u >> 52) & 0x7ffULL) - 1023;
    double m = __longlong_as_double((long long)((u & 0x000fffffffffffffULL) | 0x3ff0000000000000ULL));
    if (m > BES_SQRT2) { m = m * 0.5; e += 1; }
    double f = m - 1.0;
    double s = f / (2.0 + f);
    double z = s * s;
    double t = 0.07407407407407407;
    t = fma(t, z, 0.08);
    t = fma(t, z, 0.08695652173913043);
    t = fma(t, z, 0.09523809523809523);
    t = fma(t, z, 0.10526315789473684);
    t = fma(t, z, 0.11764705882352941);
    t = fma(t, z, 0.13333333333333333);
    t = fma(t, z, 0.15384615384615385);
    t = fma(t, z, 0.18181818181818182);
    t = fma(t, z, 0.2222222222222222);
    t = fma(t, z, 0.2857142857142857);
    t = fma(t, z, 0.4);
    t = fma(t, z, 0.6666666666666666);
    t = t * z;
    double c = s * (f - t);
    double lh = f - c;
    double ll = (f - lh) - c;
    double ed = (double)e;
    double eh = ed * BES_LN2_HI;
    double el = ed * BES_LN2_LO;
    double sh = eh + lh;
    double bb = sh - eh;
    double sl = (eh - (sh - bb)) + (lh - bb);
    sl = sl + (ll + el);
    double h = sh + sl;
    hi = h;
    lo = sl - (h - sh);
}

__device__ __forceinline__ bool is_int(double y) {
    return fabs(y) < 9007199254740992.0 ? round_nearest(y) == y : true;
}
__device__ __forceinline__ bool is_odd_int(double y) {
    if (!(fabs(y) < 9007199254740992.0)) return false;
    if (round_nearest(y) != y) return false;
    double h = y * 0.5;
    return round_nearest(h) != h;
}

__device__ __forceinline__ double pow(double x, double y) {
    const double inf = __longlong_as_double(0x7ff0000000000000LL);
    if (y == 0.0) return 1.0;
    if (x == 1.0) return 1.0;
    if (x != x || y != y) return x + y;
    double sign = 1.0;
    if (x < 0.0) {
        if (isinf(y)) { x = -x; }
        else if (!is_int(y)) return __longlong_as_double(0x7ff8000000000000LL);
        else { if (is_odd_int(y)) sign = -1.0; x = -x; }
    }
    if (isinf(y)) {
        if (x == 1.0) return 1.0;
        if ((x < 1.0) == (y > 0.0)) return 0.0;
        return inf;
    }
    if (x == 0.0) return y > 0.0 ? sign * 0.0 : sign * inf;
    if (isinf(x)) return y > 0.0 ? sign * inf : sign * 0.0;
    double lh, ll;
    log_hl(x, lh, ll);
    double ph = y * lh;
    double pl = fma(y, lh, -ph);
    pl = fma(y, ll, pl);
    return sign * exp_ab(ph, pl);
}

/* (1/x)^y as exp(-y log x): no reciprocal on the dependency chain and no
 * rounding of 1/x; positive finite x and finite nonzero y, anything else
 * goes through pow(1/x, y) */
__device__ __forceinline__ double pow_recip(double x, double y) {
    if (!(x > 0.0 && x < 1.0e300 && x > 1.0e-300) || !(fabs(y) < 1.0e300) || y == 0.0) return pow(1.0 / x, y);
    double lh, ll;
    log_hl(x, lh, ll);
    const double ny = -y;
    double ph = ny * lh;
    double pl = fma(ny, lh, -ph);
    pl = fma(ny, ll, pl);
    return exp_ab(ph, pl);
}

/* sin(pi x), cos(pi x) */
__device__ __forceinline__ void sincospi(double x, double& s, double& c) {
    if (!isfinite(x)) { s = __longlong_as_double(0x7ff8000000000000LL); c = s; return; }
    double n = round_nearest(x + x);
    double r = fma(-0.5, n, x);
    double z = r * r;
    double ps = 7.952054001475513e-07;
    ps = fma(ps, z, -2.1915353447830217e-05);
    ps = fma(ps, z, 0.00046630280576761255);
    ps = fma(ps, z, -0.0073704309457143504);
    ps = fma(ps, z, 0.08214588661112823);
    ps = fma(ps, z, -0.5992645293207921);
    ps = fma(ps, z, 2.5501640398773455);
    ps = fma(ps, z, -5.16771278004997);
    ps = fma(ps, z, 3.141592653589793);
    ps = ps * r;
    double pc = -1.3878952462213771e-07;
    pc = fma(pc, z, 4.303069587032947e-06);
    pc = fma(pc, z, -0.0001046381049248457);
    pc = fma(pc, z, 0.0019295743094039231);
    pc = fma(pc, z, -0.02580689139001406);
    pc = fma(pc, z, 0.2353306303588932);
    pc = fma(pc, z, -1.3352627688545895);
    pc = fma(pc, z, 4.0587121264167685);
    pc = fma(pc, z, -4.934802200544679);
    pc = fma(pc, z, 1.0);
    int q = (int)((long long)n & 3);
    if (q == 0) { s = ps; c = pc; }
    else if (q == 1) { s = pc; c = -ps; }
    else if (q == 2) { s = -ps; c = -pc; }
    else { s = -pc; c = ps; }
}

#define BES_PIO2_1 1.5707963267341256
#define BES_PIO2_2 6.077100506303966e-11
#define BES_PIO2_3 2.0222662487959506e-21
#define BES_INV_PIO2 0.6366197723675814

/* sin(x), cos(x) */
__device__ __forceinline__ void sincos(double x, double& s, double& c) {
    if (!isfinite(x)) { s = __longlong_as_double(0x7ff8000000000000LL); c = s; return; }
    double kd = round_nearest(x * BES_INV_PIO2);
    double r = fma(-kd, BES_PIO2_1, x);
    r = fma(-kd, BES_PIO2_2, r);
    r = fma(-kd, BES_PIO2_3, r);
    double z = r * r;
    double ps = -8.22063524662433e-18;
    ps = fma(ps, z, 2.8114572543455206e-15);
    ps = fma(ps, z, -7.647163731819816e-13);
    ps = fma(ps, z, 1.6059043836821613e-10);
    ps = fma(ps, z, -2.505210838544172e-08);
    ps = fma(ps, z, 2.7557319223985893e-06);
    ps = fma(ps, z, -0.0001984126984126984);
    ps = fma(ps, z, 0.008333333333333333);
    ps = fma(ps, z, -0.16666666666666666);
    ps = ps * z;
    ps = fma(ps, r, r);
    double pc = 4.110317623312165e-19;
    pc = fma(pc, z, -1.5619206968586225e-16);
    pc = fma(pc, z, 4.779477332387385e-14);
    pc = fma(pc, z, -1.1470745597729725e-11);
    pc = fma(pc, z, 2.08767569878681e-09);
    pc = fma(pc, z, -2.755731922398589e-07);
    pc = fma(pc, z, 2.48015873015873e-05);
    pc = fma(pc, z, -0.001388888888888889);
    pc = fma(pc, z, 0.041666666666666664);
    pc = fma(pc, z, -0.5);
    pc = fma(pc, z, 1.0);
    int q = (int)((long long)kd & 3);
    if (q == 0) { s = ps; c = pc; }
    else if (q == 1) { s = pc; c = -ps; }
    else if (q == 2) { s = -ps; c = -pc; }
    else { s = -pc; c = ps; }
}

}  // namespace math
}  // namespace bes

#endif
