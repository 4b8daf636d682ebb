/*
 * oracle_math.h -- TEST INFRASTRUCTURE (the oracle's own elementary functions).
 *
 * The reference calls CUDA's device `pow`, `sincospi`, `sin` and `cos`
 * (BubbleEnsemble_SystemDefinition.cuh:16-23 for the Keller-Miksis right-hand
 * side, SourceCodes/CoupledSystems_PerBlock_ExplicitRungeKutta_ErrorControllers.cuh:502-505
 * for the step-size factor).  The oracle does not reproduce those library
 * routines.  It restates the functions from textbook mathematics:
 *
 *   exp   : Cody-Waite reduction x = k ln2 + r (ln2 split into a 32-bit head
 *           and a tail), Taylor polynomial of degree 13 on |r| <= ln2/2,
 *           scaling by 2^k through the exponent field.
 *   log   : x = 2^e m, m in (sqrt(2)/2, sqrt(2)], f = m - 1,
 *           log(1+f) = 2 atanh(s) with s = f/(2+f)
 *                    = f - s (f - T(s^2)),  T(z) = sum_k 2 z^k / (2k+1),
 *           returned as a head/tail pair.
 *   pow   : exp(y log x) with the product y*log x carried as head + tail.
 *   sinpi/cospi : x = n/2 + r, |r| <= 1/4, Taylor series of sin(pi r) and
 *           cos(pi r), quadrant from n mod 4.
 *   sin/cos: Cody-Waite reduction by pi/2 split into three parts (33, 33 and
 *           53 bits), Taylor series on |r| <= pi/4.
 *
 * Every coefficient is a Taylor coefficient (1/k!, pi^k/k!, 2/(2k+1)) or a
 * digit split of pi/2 and ln 2, computed in exact rational / 80-digit decimal
 * arithmetic and rounded to the nearest double.  Only +, -, *, /, fma and
 * exponent-field manipulation are used, so the CUDA kernel's separately
 * written copy of the same algorithm (compiled without implicit FMA
 * contraction) returns bit-identical results.  The tests check these
 * functions against the C library to a few ulp.
 *
 * Compile with -ffp-contract=off: every fused multiply-add below is explicit.
 */
#ifndef BES_ORACLE_MATH_H
#define BES_ORACLE_MATH_H

#include <cmath>
#include <cstdint>
#include <cstring>

namespace oracle_math {

static inline uint64_t bits_of(double x) { uint64_t u; std::memcpy(&u, &x, 8); return u; }
static inline double from_bits(uint64_t u) { double x; std::memcpy(&x, &u, 8); return x; }

/* round to nearest integer (ties to even) for |x| < 2^51; larger |x| are integers already */
static inline double rint_nearest(double x) {
    const double M = 6755399441055744.0; /* 1.5 * 2^52 */
    if (std::fabs(x) >= 2251799813685248.0) return x;
    double t = x + M;
    return t - M;
}

/* x * 2^k for x in [0.5, 2) */
static inline double scale_pow2(double x, int k) {
    if (k > 1023) {
        x = x * from_bits((uint64_t)(1023 + 1023) << 52);
        k -= 1023;
        if (k > 1023) return x * INFINITY;
        return x * from_bits((uint64_t)(k + 1023) << 52);
    }
    if (k < -1022) {
        x = x * from_bits((uint64_t)(-1000 + 1023) << 52);
        k += 1000;
        if (k < -1022) return x * 0.0;
        return x * from_bits((uint64_t)(k + 1023) << 52);
    }
    return x * from_bits((uint64_t)(k + 1023) << 52);
}

static const double LN2_HI = 0.6931471806019545;       /* ln 2 rounded to 32 significant bits */
static const double LN2_LO = -4.2009150726810846e-11;  /* ln 2 - LN2_HI */
static const double INV_LN2 = 1.4426950408889634;
static const double SQRT2 = 1.4142135623730951;

/* exp(a + b), |b| much smaller than 1 (b is a correction term) */
static inline double exp_ab(double a, double b) {
    if (a != a) return a;
    if (a > 709.8) return INFINITY;
    if (a < -745.2) return 0.0;
    double kd = rint_nearest(a * INV_LN2);
    double r = std::fma(-kd, LN2_HI, a);
    r = std::fma(-kd, LN2_LO, r);
    r = r + b;
    double p = 1.6059043836821613e-10;            /* 1/13! */
    p = std::fma(p, r, 2.08767569878681e-09);     /* 1/12! */
    p = std::fma(p, r, 2.505210838544172e-08);    /* 1/11! */
    p = std::fma(p, r, 2.755731922398589e-07);    /* 1/10! */
    p = std::fma(p, r, 2.7557319223985893e-06);   /* 1/9!  */
    p = std::fma(p, r, 2.48015873015873e-05);     /* 1/8!  */
    p = std::fma(p, r, 0.0001984126984126984);    /* 1/7!  */
    p = std::fma(p, r, 0.001388888888888889);     /* 1/6!  */
    p = std::fma(p, r, 0.008333333333333333);     /* 1/5!  */
    p = std::fma(p, r, 0.041666666666666664);     /* 1/4!  */
    p = std::fma(p, r, 0.16666666666666666);      /* 1/3!  */
    p = std::fma(p, r, 0.5);                      /* 1/2!  */
    p = std::fma(p, r, 1.0);
    p = std::fma(p, r, 1.0);
    return scale_pow2(p, (int)kd);
}

static inline double exp(double a) { return exp_ab(a, 0.0); }

/* log(x) = hi + lo for finite x > 0 */
static inline void log_hl(double x, double* hi, double* lo) {
    int e = 0;
    if (x < 2.2250738585072014e-308) { x = x * 18014398509481984.0; e = -54; } /* 2^54 */
    uint64_t u = bits_of(x);
    e += (int)((u >> 52) & 0x7ff) - 1023;
    double m = from_bits((u & 0x000fffffffffffffULL) | 0x3ff0000000000000ULL);
    if (m > SQRT2) { m = m * 0.5; e += 1; }
    double f = m - 1.0;
    double s = f / (2.0 + f);
    double z = s * s;
    double t = 0.07407407407407407;          /* 2/27 */
    t = std::fma(t, z, 0.08);                /* 2/25 */
    t = std::fma(t, z, 0.08695652173913043); /* 2/23 */
    t = std::fma(t, z, 0.09523809523809523); /* 2/21 */
    t = std::fma(t, z, 0.10526315789473684); /* 2/19 */
    t = std::fma(t, z, 0.11764705882352941); /* 2/17 */
    t = std::fma(t, z, 0.13333333333333333); /* 2/15 */
    t = std::fma(t, z, 0.15384615384615385); /* 2/13 */
    t = std::fma(t, z, 0.18181818181818182); /* 2/11 */
    t = std::fma(t, z, 0.2222222222222222);  /* 2/9  */
    t = std::fma(t, z, 0.2857142857142857);  /* 2/7  */
    t = std::fma(t, z, 0.4);                 /* 2/5  */
    t = std::fma(t, z, 0.6666666666666666);  /* 2/3  */
    t = t * z;
    double c = s * (f - t);
    double lh = f - c;
    double ll = (f - lh) - c;
    double ed = (double)e;
    double eh = ed * LN2_HI;
    double el = ed * LN2_LO;
    double sh = eh + lh;
    double bb = sh - eh;
    double sl = (eh - (sh - bb)) + (lh - bb);
    sl = sl + (ll + el);
    double h = sh + sl;
    *hi = h;
    *lo = sl - (h - sh);
}

static inline double log(double x) {
    if (x != x || x < 0.0) return NAN;
    if (x == 0.0) return -INFINITY;
    if (x == INFINITY) return INFINITY;
    double h, l;
    log_hl(x, &h, &l);
    return h + l;
}

static inline bool is_integer(double y) { return std::fabs(y) < 9007199254740992.0 ? rint_nearest(y) == y : true; }
static inline bool is_odd_integer(double y) {
    if (!(std::fabs(y) < 9007199254740992.0)) return false;
    if (rint_nearest(y) != y) return false;
    double h = y * 0.5;
    return rint_nearest(h) != h;
}

/* x^y with C99 special cases */
static inline double pow(double x, double y) {
    if (y == 0.0) return 1.0;
    if (x == 1.0) return 1.0;
    if (x != x || y != y) return x + y;
    double sign = 1.0;
    if (x < 0.0) {
        if (std::isinf(y)) { x = -x; }
        else if (!is_integer(y)) return NAN;
        else { if (is_odd_integer(y)) sign = -1.0; x = -x; }
    }
    if (std::isinf(y)) {
        if (x == 1.0) return 1.0;
        if ((x < 1.0) == (y > 0.0)) return 0.0;
        return INFINITY;
    }
    if (x == 0.0) return y > 0.0 ? sign * 0.0 : sign * INFINITY;
    if (std::isinf(x)) return y > 0.0 ? sign * INFINITY : sign * 0.0;
    double lh, ll;
    log_hl(x, &lh, &ll);
    double ph = y * lh;
    double pl = std::fma(y, lh, -ph);
    pl = std::fma(y, ll, pl);
    return sign * exp_ab(ph, pl);
}

/* (1/x)^y as exp(-y log x); positive finite x and finite nonzero y, anything
 * else through pow(1/x, y) (device: bes_math.cuh pow_recip) */
static inline double pow_recip(double x, double y) {
    if (!(x > 0.0 && x < 1.0e300 && x > 1.0e-300) || !(std::fabs(y) < 1.0e300) || y == 0.0) return pow(1.0 / x, y);
    double lh, ll;
    log_hl(x, &lh, &ll);
    const double ny = -y;
    double ph = ny * lh;
    double pl = std::fma(ny, lh, -ph);
    pl = std::fma(ny, ll, pl);
    return exp_ab(ph, pl);
}

/* sin(pi x), cos(pi x) */
static inline void sincospi(double x, double* s, double* c) {
    if (!std::isfinite(x)) { *s = NAN; *c = NAN; return; }
    double n = rint_nearest(x + x);
    double r = std::fma(-0.5, n, x);
    double z = r * r;
    double ps = 7.952054001475513e-07;
    ps = std::fma(ps, z, -2.1915353447830217e-05);
    ps = std::fma(ps, z, 0.00046630280576761255);
    ps = std::fma(ps, z, -0.0073704309457143504);
    ps = std::fma(ps, z, 0.08214588661112823);
    ps = std::fma(ps, z, -0.5992645293207921);
    ps = std::fma(ps, z, 2.5501640398773455);
    ps = std::fma(ps, z, -5.16771278004997);
    ps = std::fma(ps, z, 3.141592653589793);
    ps = ps * r;
    double pc = -1.3878952462213771e-07;
    pc = std::fma(pc, z, 4.303069587032947e-06);
    pc = std::fma(pc, z, -0.0001046381049248457);
    pc = std::fma(pc, z, 0.0019295743094039231);
    pc = std::fma(pc, z, -0.02580689139001406);
    pc = std::fma(pc, z, 0.2353306303588932);
    pc = std::fma(pc, z, -1.3352627688545895);
    pc = std::fma(pc, z, 4.0587121264167685);
    pc = std::fma(pc, z, -4.934802200544679);
    pc = std::fma(pc, z, 1.0);
    int q = (int)((int64_t)n & 3);
    switch (q) {
        case 0: *s = ps; *c = pc; break;
        case 1: *s = pc; *c = -ps; break;
        case 2: *s = -ps; *c = -pc; break;
        default: *s = -pc; *c = ps; break;
    }
}

static const double PIO2_1 = 1.5707963267341256;      /* pi/2 rounded to 33 bits */
static const double PIO2_2 = 6.077100506303966e-11;   /* next 33 bits */
static const double PIO2_3 = 2.0222662487959506e-21;  /* remainder */
static const double INV_PIO2 = 0.6366197723675814;

/* sin(x), cos(x) for |x| < 2^30 (larger arguments lose accuracy but stay deterministic) */
static inline void sincos(double x, double* s, double* c) {
    if (!std::isfinite(x)) { *s = NAN; *c = NAN; return; }
    double kd = rint_nearest(x * INV_PIO2);
    double r = std::fma(-kd, PIO2_1, x);
    r = std::fma(-kd, PIO2_2, r);
    r = std::fma(-kd, PIO2_3, r);
    double z = r * r;
    double ps = -8.22063524662433e-18;
    ps = std::fma(ps, z, 2.8114572543455206e-15);
    ps = std::fma(ps, z, -7.647163731819816e-13);
    ps = std::fma(ps, z, 1.6059043836821613e-10);
    ps = std::fma(ps, z, -2.505210838544172e-08);
    ps = std::fma(ps, z, 2.7557319223985893e-06);
    ps = std::fma(ps, z, -0.0001984126984126984);
    ps = std::fma(ps, z, 0.008333333333333333);
    ps = std::fma(ps, z, -0.16666666666666666);
    ps = ps * z;
    ps = std::fma(ps, r, r);
    double pc = 4.110317623312165e-19;
    pc = std::fma(pc, z, -1.5619206968586225e-16);
    pc = std::fma(pc, z, 4.779477332387385e-14);
    pc = std::fma(pc, z, -1.1470745597729725e-11);
    pc = std::fma(pc, z, 2.08767569878681e-09);
    pc = std::fma(pc, z, -2.755731922398589e-07);
    pc = std::fma(pc, z, 2.48015873015873e-05);
    pc = std::fma(pc, z, -0.001388888888888889);
    pc = std::fma(pc, z, 0.041666666666666664);
    pc = std::fma(pc, z, -0.5);
    pc = std::fma(pc, z, 1.0);
    int q = (int)((int64_t)kd & 3);
    switch (q) {
        case 0: *s = ps; *c = pc; break;
        case 1: *s = pc; *c = -ps; break;
        case 2: *s = -ps; *c = -pc; break;
        default: *s = -pc; *c = ps; break;
    }
}

}  // namespace oracle_math

#endif
