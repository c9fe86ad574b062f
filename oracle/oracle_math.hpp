// oracle/oracle_math.hpp -- TEST INFRASTRUCTURE (the CPU oracle). Only tests/, __graft_entry__.smoke() and the
// cpu_baseline / reference legs of bench.py use anything under oracle/; the product never does.
//
// Scalar arithmetic of the oracle with Julia's Float64 semantics:
//  * `jl_max` / `jl_min`: Julia's `max` / `min` for floats (NaN propagates; max prefers +0, min prefers -0);
//  * `_sin` / `_cos` of src/Systems/standard_map.jl:13-14: non-finite input gives `x - x` (NaN);
//  * two transcendental back ends, chosen per call:
//      MATH_LIBM     - glibc sin / cos / log, the closest stand-in for Julia's Base libm (Julia 1.13.2 is absent here);
//      MATH_PORTABLE - the oracle's own sin / cos / log: Cody-Waite reduction by pi/2 with a three-part constant
//                      (Cody and Waite 1980), Taylor polynomials of sin and cos on [-pi/4, pi/4], and the fdlibm-form
//                      identity log(1+f) = f - f^2/2 + s (f^2/2 + R(s^2)), s = f/(2+f), R the atanh series. Written
//                      with explicit fma only, so it gives the same bits on any IEEE binary64 machine with fma.
// Build with -ffp-contract=off: no implicit fusion anywhere (Julia does not contract a*b+c either).
#pragma once

#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>

#include "oracle_constants.hpp"

namespace orc {

enum MathMode { MATH_PORTABLE = 0, MATH_LIBM = 1 };

inline bool isfin(double x) { return std::isfinite(x); }

// Julia: max(x, y) for IEEE floats -- NaN if either is NaN, +0 preferred over -0.
inline double jl_max(double x, double y) {
    if (std::isnan(x) || std::isnan(y)) return x - y;
    if (x == y) return std::signbit(x) ? y : x;
    return x > y ? x : y;
}
// Julia: min(x, y) -- NaN if either is NaN, -0 preferred over +0.
inline double jl_min(double x, double y) {
    if (std::isnan(x) || std::isnan(y)) return x - y;
    if (x == y) return std::signbit(x) ? x : y;
    return x < y ? x : y;
}

inline uint64_t bits_of(double x) { uint64_t b; std::memcpy(&b, &x, 8); return b; }
inline double of_bits(uint64_t b) { double x; std::memcpy(&x, &b, 8); return x; }

// ---- portable sin / cos (both from one reduction) ---------------------------------------------------------------
inline void p_sincos(double x, double* sn, double* cs) {
    if (!isfin(x)) { *sn = x - x; *cs = x - x; return; }
    if (x == 0.0) { *sn = x; *cs = 1.0; return; }              // keeps sin(-0) = -0
    const double k = std::nearbyint(x * CL_TWO_OVER_PI);
    double r = std::fma(-k, CL_PIO2_1, x);                       // exact: |r| < 2, multiple of ulp(k * P1)
    r = std::fma(-k, CL_PIO2_2, r);
    r = std::fma(-k, CL_PIO2_3, r);
    const double z = r * r;
    double ps = CL_SIN_T17;
    ps = std::fma(ps, z, CL_SIN_T15);
    ps = std::fma(ps, z, CL_SIN_T13);
    ps = std::fma(ps, z, CL_SIN_T11);
    ps = std::fma(ps, z, CL_SIN_T9);
    ps = std::fma(ps, z, CL_SIN_T7);
    ps = std::fma(ps, z, CL_SIN_T5);
    ps = std::fma(ps, z, CL_SIN_T3);
    const double s = std::fma(r * z, ps, r);
    double pc = CL_COS_T16;
    pc = std::fma(pc, z, CL_COS_T14);
    pc = std::fma(pc, z, CL_COS_T12);
    pc = std::fma(pc, z, CL_COS_T10);
    pc = std::fma(pc, z, CL_COS_T8);
    pc = std::fma(pc, z, CL_COS_T6);
    pc = std::fma(pc, z, CL_COS_T4);
    pc = std::fma(pc, z, CL_COS_T2);
    const double c = std::fma(z, pc, 1.0);
    const double q = k - 4.0 * std::floor(k * 0.25);            // quadrant, exact for every integral k
    if (q == 0.0) { *sn = s; *cs = c; }
    else if (q == 1.0) { *sn = c; *cs = -s; }
    else if (q == 2.0) { *sn = -s; *cs = -c; }
    else { *sn = -c; *cs = s; }
}

// ---- portable natural logarithm ------------------------------------------------------------------------------------
inline double p_log(double x) {
    if (std::isnan(x)) return x;
    if (x < 0.0) return std::numeric_limits<double>::quiet_NaN();
    if (x == 0.0) return -std::numeric_limits<double>::infinity();
    if (x == std::numeric_limits<double>::infinity()) return x;
    double e = 0.0;
    uint64_t b = bits_of(x);
    if (x < std::numeric_limits<double>::min()) { b = bits_of(x * 0x1p54); e = -54.0; }
    e += static_cast<double>(static_cast<int64_t>((b >> 52) & 0x7ff) - 1023);
    double m = of_bits((b & 0x000fffffffffffffULL) | 0x3ff0000000000000ULL);   // [1, 2)
    if (m > CL_SQRT2) { m = m * 0.5; e = e + 1.0; }                              // [sqrt(1/2), sqrt(2)]
    const double f = m - 1.0;
    const double s = f / (2.0 + f);
    const double z = s * s;
    double R = CL_LOG_T9;
    R = std::fma(R, z, CL_LOG_T8);
    R = std::fma(R, z, CL_LOG_T7);
    R = std::fma(R, z, CL_LOG_T6);
    R = std::fma(R, z, CL_LOG_T5);
    R = std::fma(R, z, CL_LOG_T4);
    R = std::fma(R, z, CL_LOG_T3);
    R = std::fma(R, z, CL_LOG_T2);
    R = std::fma(R, z, CL_LOG_T1);
    R = R * z;
    const double hfsq = 0.5 * f * f;
    return e * CL_LN2_HI - ((hfsq - (s * (hfsq + R) + e * CL_LN2_LO)) - f);
}

// ---- portable exp: k = rint(x / ln 2), r = (x - k LN2_HI) - k LN2_LO (the first product exact), the Taylor
// polynomial of exp(r) to r^13 in Horner form, then the scaling by 2^k in at most two exact-or-once-rounded products.
inline double p_pow2(int k) { return of_bits(static_cast<uint64_t>(k + 1023) << 52); }   // -1022 <= k <= 1023
inline double p_exp(double x) {
    if (std::isnan(x)) return x;
    if (x > 709.782712893384) return std::numeric_limits<double>::infinity();
    if (x < -745.1332191019412) return 0.0;
    const double k = std::rint(x * CL_INV_LN2);
    const double r = (x - k * CL_LN2_HI) - k * CL_LN2_LO;
    double p = CL_EXP_T13;
    p = std::fma(p, r, CL_EXP_T12);
    p = std::fma(p, r, CL_EXP_T11);
    p = std::fma(p, r, CL_EXP_T10);
    p = std::fma(p, r, CL_EXP_T9);
    p = std::fma(p, r, CL_EXP_T8);
    p = std::fma(p, r, CL_EXP_T7);
    p = std::fma(p, r, CL_EXP_T6);
    p = std::fma(p, r, CL_EXP_T5);
    p = std::fma(p, r, CL_EXP_T4);
    p = std::fma(p, r, CL_EXP_T3);
    p = std::fma(p, r, CL_EXP_T2);
    p = std::fma(p, r, 1.0);
    p = std::fma(p, r, 1.0);
    const int ki = static_cast<int>(k);
    if (ki > 1023) return (p * p_pow2(1023)) * p_pow2(ki - 1023);
    if (ki >= -1022) return p * p_pow2(ki);
    return (p * p_pow2(ki + 1000)) * p_pow2(-1000);
}

// ---- portable atan2: the octant reduction to z = min / max in [0, 1], atan(z) = atan(c) + atan(u) with c = k / 16
// the nearest table point and u = (z - c) / (1 + z c), |u| <= 1/32, atan(u) by its Taylor polynomial to u^13, then
// pi / 2 - a and pi - a with split constants; the C99 special cases for zeros and infinities.
constexpr double P_ATAN_HI[17] = {CL_ATAN_HI_0, CL_ATAN_HI_1, CL_ATAN_HI_2, CL_ATAN_HI_3, CL_ATAN_HI_4, CL_ATAN_HI_5,
                                  CL_ATAN_HI_6, CL_ATAN_HI_7, CL_ATAN_HI_8, CL_ATAN_HI_9, CL_ATAN_HI_10, CL_ATAN_HI_11,
                                  CL_ATAN_HI_12, CL_ATAN_HI_13, CL_ATAN_HI_14, CL_ATAN_HI_15, CL_ATAN_HI_16};
constexpr double P_ATAN_LO[17] = {CL_ATAN_LO_0, CL_ATAN_LO_1, CL_ATAN_LO_2, CL_ATAN_LO_3, CL_ATAN_LO_4, CL_ATAN_LO_5,
                                  CL_ATAN_LO_6, CL_ATAN_LO_7, CL_ATAN_LO_8, CL_ATAN_LO_9, CL_ATAN_LO_10, CL_ATAN_LO_11,
                                  CL_ATAN_LO_12, CL_ATAN_LO_13, CL_ATAN_LO_14, CL_ATAN_LO_15, CL_ATAN_LO_16};
inline double p_atan01(double z) {
    const int k = static_cast<int>(std::rint(z * 16.0));
    const double c = k * 0.0625;
    const double u = (z - c) / (1.0 + z * c);
    const double u2 = u * u;
    double q = CL_ATAN_T13;
    q = std::fma(q, u2, CL_ATAN_T11);
    q = std::fma(q, u2, CL_ATAN_T9);
    q = std::fma(q, u2, CL_ATAN_T7);
    q = std::fma(q, u2, CL_ATAN_T5);
    q = std::fma(q, u2, CL_ATAN_T3);
    const double at = std::fma(u * u2, q, u);
    return P_ATAN_HI[k] + (at + P_ATAN_LO[k]);
}
inline double p_atan2(double y, double x) {
    if (std::isnan(x) || std::isnan(y)) return x + y;
    if (std::isinf(y)) {
        const double a = std::isinf(x) ? (x > 0 ? CL_PIO2_1 * 0.5 : (CL_PI_HI - CL_PIO2_1 * 0.5) + CL_PI_LO)
                                       : CL_PIO2_1;
        return std::copysign(a, y);
    }
    if (std::isinf(x)) return std::copysign(x > 0 ? 0.0 : CL_PI_HI, y);
    if (y == 0.0) return std::signbit(x) ? std::copysign(CL_PI_HI, y) : y;
    if (x == 0.0) return std::copysign(CL_PIO2_1, y);
    const double ax = std::fabs(x), ay = std::fabs(y);
    const bool swap = ay > ax;
    double a = p_atan01(swap ? ax / ay : ay / ax);
    if (swap) a = (CL_PIO2_1 - a) + CL_PIO2_2;
    if (x < 0.0) a = (CL_PI_HI - a) + CL_PI_LO;
    return y < 0.0 ? -a : a;
}

template <int MM> struct Math;
template <> struct Math<MATH_PORTABLE> {
    static void sincos(double x, double* s, double* c) { p_sincos(x, s, c); }
    static double sin(double x) { double s, c; p_sincos(x, &s, &c); return s; }
    static double cos(double x) { double s, c; p_sincos(x, &s, &c); return c; }
    static double log(double x) { return p_log(x); }
    static double exp(double x) { return p_exp(x); }
    static double atan2(double y, double x) { return p_atan2(y, x); }
};
template <> struct Math<MATH_LIBM> {
    static void sincos(double x, double* s, double* c) {
        if (!isfin(x)) { *s = x - x; *c = x - x; return; }
        *s = std::sin(x); *c = std::cos(x);
    }
    static double sin(double x) { return isfin(x) ? std::sin(x) : x - x; }
    static double cos(double x) { return isfin(x) ? std::cos(x) : x - x; }
    static double log(double x) { return std::log(x); }
    static double exp(double x) { return std::exp(x); }
    static double atan2(double y, double x) { return std::atan2(y, x); }
};

}  // namespace orc
