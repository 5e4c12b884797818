// Exponential, logarithm and power of the ground friction's Stribeck curve (static_world.cpp:41-44).
//
// libm's float exp/pow (what the reference links) are not correctly rounded in every case, so no GPU function can
// match them bit for bit. These functions fix one result instead: Cody-Waite range reduction x = k ln2 + r, exp(r)
// by its Taylor series to degree 13 (|r| <= ln2/2), log m = 2 atanh((m - 1)/(m + 1)) by its series to degree 27,
// pow x^y = exp(y log x), all in double precision and rounded once to float. Compiled without FMA contraction, every
// operation rounds once, so any IEEE machine computes the same bits: the CPU oracle evaluates the same operations
// (oracle/orc_math.h) and so the GPU's trajectories are bitwise the oracle's. Against libm the results agree to within
// one unit in the last place.
#pragma once

namespace blg {

__device__ __forceinline__ double bl_exp_d(double x) {
    if (x != x) return x;
    if (x > 700.0) return __longlong_as_double(0x7ff0000000000000LL);
    if (x < -700.0) return 0.0;
    const double kd = floor(x * 0x1.71547652b82fep+0 + 0.5);   // nearest integer to x / ln2
    const double r = (x - kd * 0x1.62e42fefa3800p-1) - kd * 0x1.ef35793c76730p-45; // x - k ln2 (ln2 in two parts)
    double p = 0x1.6124613a86d09p-33;                            // 1/13!
    p = p * r + 0x1.1eed8eff8d898p-29;
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

__device__ __forceinline__ double bl_log_d(double x) { // x > 0, finite
    int e;
    double m = frexp(x, &e);
    if (m < 0x1.6a09e667f3bcdp-1) m = m * 2.0, e = e - 1;     // m in [sqrt(1/2), sqrt(2))
    const double s = (m - 1.0) / (m + 1.0);
    const double s2 = s * s;
    double t = 0x1.2f684bda12f68p-5;                             // 1/27
    t = t * s2 + 0x1.47ae147ae147bp-5;
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
    return ed * 0x1.62e42fefa3800p-1 + (ed * 0x1.ef35793c76730p-45 + 2.0 * s * t);
}

__device__ __forceinline__ float bl_expf(float x) { return (float)bl_exp_d((double)x); }

__device__ __forceinline__ float bl_powf(float x, float y) { // the friction curve's x >= 0
    if (y == 0.0f) return 1.0f;
    if (x != x || y != y || x < 0.0f) return __int_as_float(0x7fc00000);
    if (x == 0.0f) return y > 0.0f ? 0.0f : __int_as_float(0x7f800000);
    if (isinf(x)) return y > 0.0f ? __int_as_float(0x7f800000) : 0.0f;
    return (float)bl_exp_d((double)y * bl_log_d((double)x));
}

} // namespace blg
