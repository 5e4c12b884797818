/* Test infrastructure only: the portable exponential, logarithm and power of the oracle.
 *
 * The reference calls libm's expf and powf in the ground contact's Stribeck friction (static_world.cpp:41-44). libm's
 * float results are not correctly rounded in every case, so no other implementation can match them bit for bit. The
 * oracle therefore uses these functions - written from the mathematics: Cody-Waite range reduction x = k ln2 + r,
 * exp(r) by its Taylor series to degree 13 (|r| <= ln2/2: error below 1e-17), log m = 2 atanh((m - 1)/(m + 1)) by its
 * series to degree 27, pow x^y = exp(y log x); all in double precision, rounded once to float - and the GPU kernels
 * evaluate the very same operations (beamlab_b200/csrc/bl_math.cuh), as does the parity build of the reference
 * (oracle/ref_libm.c replaces its expf / powf). Against libm they agree to within one unit in the last place.
 * Built without FMA contraction: each operation rounds once, identically on every IEEE machine. */
#ifndef BEAMLAB_ORC_MATH_H
#define BEAMLAB_ORC_MATH_H

#include <math.h>

static const double ORC_LN2_HI = 0x1.62e42fefa3800p-1;  /* ln 2 to 42 bits: k * ORC_LN2_HI is exact */
static const double ORC_LN2_LO = 0x1.ef35793c76730p-45; /* ln 2 - ORC_LN2_HI */
static const double ORC_INV_LN2 = 0x1.71547652b82fep+0;
static const double ORC_SQRT_HALF = 0x1.6a09e667f3bcdp-1;

/* e^x, x finite and |x| <= 700 */
static inline double orc_exp_core(double x) {
    const double kd = floor(x * ORC_INV_LN2 + 0.5);
    const double r = (x - kd * ORC_LN2_HI) - kd * ORC_LN2_LO;
    double p = 0x1.6124613a86d09p-33;              /* 1/13! */
    p = p * r + 0x1.1eed8eff8d898p-29;             /* 1/12! */
    p = p * r + 0x1.ae64567f544e4p-26;
    p = p * r + 0x1.27e4fb7789f5cp-22;
    p = p * r + 0x1.71de3a556c734p-19;
    p = p * r + 0x1.a01a01a01a01ap-16;
    p = p * r + 0x1.a01a01a01a01ap-13;
    p = p * r + 0x1.6c16c16c16c17p-10;
    p = p * r + 0x1.1111111111111p-7;
    p = p * r + 0x1.5555555555555p-5;
    p = p * r + 0x1.5555555555555p-3;
    p = p * r + 0x1.0000000000000p-1;
    p = p * r + 1.0;
    p = p * r + 1.0;
    return ldexp(p, (int)kd);
}

static inline double orc_exp_d(double x) {
    if (x != x) return x;
    if (x > 700.0) return INFINITY;
    if (x < -700.0) return 0.0;
    return orc_exp_core(x);
}

/* natural log, x > 0 finite */
static inline double orc_log_d(double x) {
    int e;
    double m = frexp(x, &e);
    if (m < ORC_SQRT_HALF) m = m * 2.0, e = e - 1;
    const double s = (m - 1.0) / (m + 1.0);
    const double s2 = s * s;
    double t = 0x1.2f684bda12f68p-5;               /* 1/27 */
    t = t * s2 + 0x1.47ae147ae147bp-5;             /* 1/25 */
    t = t * s2 + 0x1.642c8590b2164p-5;
    t = t * s2 + 0x1.8618618618618p-5;
    t = t * s2 + 0x1.af286bca1af28p-5;
    t = t * s2 + 0x1.e1e1e1e1e1e1ep-5;
    t = t * s2 + 0x1.1111111111111p-4;
    t = t * s2 + 0x1.3b13b13b13b14p-4;
    t = t * s2 + 0x1.745d1745d1746p-4;
    t = t * s2 + 0x1.c71c71c71c71cp-4;
    t = t * s2 + 0x1.2492492492492p-3;
    t = t * s2 + 0x1.999999999999ap-3;
    t = t * s2 + 0x1.5555555555555p-2;
    t = t * s2 + 1.0;
    const double ed = (double)e;
    return ed * ORC_LN2_HI + (ed * ORC_LN2_LO + 2.0 * s * t);
}

static inline float orc_expf(float x) { return (float)orc_exp_d((double)x); }

/* x^y for the friction curve: x >= 0 */
static inline float orc_powf(float x, float y) {
    if (y == 0.0f) return 1.0f;
    if (x != x || y != y || x < 0.0f) return NAN;
    if (x == 0.0f) return y > 0.0f ? 0.0f : INFINITY;
    if (isinf(x)) return y > 0.0f ? INFINITY : 0.0f;
    return (float)orc_exp_d((double)y * orc_log_d((double)x));
}

#endif
