// cl_math.cuh -- scalar arithmetic of the orbit kernels with Julia's Float64 semantics.
//
// Every kernel translation unit is compiled with -fmad=false: nothing is fused unless written as fma(), exactly as
// Julia contracts nothing (src/Foundation/product.jl:9-20 makes the frame product's fusion explicit). The Float32
// tangent path of the mixed kernels writes its fusions as __fmaf_rn() where it wants them.
//
// Transcendentals (Julia's Base libm has no device counterpart):
//   cl_sincos: Cody-Waite reduction by pi/2 with a three-part constant (Cody and Waite 1980): k = rint(x 2/pi),
//              r = ((x - k P1) - k P2) - k P3 each step one fma (the first is exact), then the Taylor polynomials of
//              sin (to x^17) and cos (to x^16) on [-pi/4, pi/4] in Horner form, and the quadrant of k. About 1 ulp
//              for |x| < 2^30; non-finite input gives NaN like `_sin` / `_cos` (src/Systems/standard_map.jl:13-14).
//   cl_log:    x = m 2^e with m in [sqrt(1/2), sqrt(2)], f = m - 1, s = f / (2 + f), and the identity
//              log(1 + f) = f - f^2/2 + s (f^2/2 + R(s^2)), R the atanh series 2z/3 + 2z^2/5 + ... to z^9, plus e ln 2
//              with ln 2 split so that e LN2_HI is exact.
//   cl_exp, cl_atan2: see their definitions below (Taylor polynomials after Cody-Waite / table reduction).
// The constants come from chaos_b200/csrc/derive_constants.py (mathematical definitions, rounded once).
#pragma once

#include <cstdint>

#include "cl_constants.h"

namespace cl {

__device__ __forceinline__ bool isfin(double x) { return isfinite(x); }
__device__ __forceinline__ bool isfin(float x) { return isfinite(x); }

// Julia max / min for IEEE floats: NaN if either is NaN; max prefers +0, min prefers -0.
template <typename T>
__device__ __forceinline__ T jl_max(T x, T y) {
    if (isnan(x) || isnan(y)) return x - y;
    if (x == y) return signbit(x) ? y : x;
    return x > y ? x : y;
}
template <typename T>
__device__ __forceinline__ T jl_min(T x, T y) {
    if (isnan(x) || isnan(y)) return x - y;
    if (x == y) return signbit(x) ? x : y;
    return x < y ? x : y;
}

__device__ __forceinline__ void cl_sincos(double x, double* sn, double* cs) {
    if (!isfin(x)) { *sn = x - x; *cs = x - x; return; }
    if (x == 0.0) { *sn = x; *cs = 1.0; return; }
    const double k = rint(x * CL_TWO_OVER_PI);
    double r = fma(-k, CL_PIO2_1, x);
    r = fma(-k, CL_PIO2_2, r);
    r = fma(-k, CL_PIO2_3, r);
    const double z = r * r;
    double ps = CL_SIN_T17;
    ps = fma(ps, z, CL_SIN_T15);
    ps = fma(ps, z, CL_SIN_T13);
    ps = fma(ps, z, CL_SIN_T11);
    ps = fma(ps, z, CL_SIN_T9);
    ps = fma(ps, z, CL_SIN_T7);
    ps = fma(ps, z, CL_SIN_T5);
    ps = fma(ps, z, CL_SIN_T3);
    const double s = fma(r * z, ps, r);
    double pc = CL_COS_T16;
    pc = fma(pc, z, CL_COS_T14);
    pc = fma(pc, z, CL_COS_T12);
    pc = fma(pc, z, CL_COS_T10);
    pc = fma(pc, z, CL_COS_T8);
    pc = fma(pc, z, CL_COS_T6);
    pc = fma(pc, z, CL_COS_T4);
    pc = fma(pc, z, CL_COS_T2);
    const double c = fma(z, pc, 1.0);
    const double q = k - 4.0 * floor(k * 0.25);
    if (q == 0.0) { *sn = s; *cs = c; }
    else if (q == 1.0) { *sn = c; *cs = -s; }
    else if (q == 2.0) { *sn = -s; *cs = -c; }
    else { *sn = -c; *cs = s; }
}
// ---- split evaluation for the mixed kernels ------------------------------------------------------------------------
// The same reduction as cl_sincos, then only the polynomial one Float64 value needs (the quadrant picks sin- or
// cos-form coefficients), so sin(x) or cos(x) comes out bit-identical to cl_sincos at about half the FP64 work;
// the complementary function comes in Float32 from the same reduced argument (Taylor to x^11 / x^10, ~1 ulp of
// float), for the Float32 tangent entries.
struct Reduced { double r, z, x; int q; };
__device__ __forceinline__ Reduced cl_reduce(double x) {
    Reduced w;
    w.x = x;
    const double k = rint(x * CL_TWO_OVER_PI);
    double r = fma(-k, CL_PIO2_1, x);
    r = fma(-k, CL_PIO2_2, r);
    r = fma(-k, CL_PIO2_3, r);
    w.r = r;
    w.z = r * r;
    // k - 4 floor(k / 4) of cl_sincos, from the integer: k is integral, so its two's-complement low bits are that
    // remainder for every |k| < 2^63 (a non-finite x gives a NaN r and the quadrant does not matter)
    w.q = static_cast<int>(static_cast<long long>(k) & 3);
    return w;
}
// cos-form (cosf = true) or sin-form polynomial of the reduced argument, exactly as cl_sincos evaluates it.
__device__ __forceinline__ double cl_poly(const Reduced& w, bool cosf) {
    const double z = w.z;
    double p = cosf ? CL_COS_T16 : CL_SIN_T17;
    p = fma(p, z, cosf ? CL_COS_T14 : CL_SIN_T15);
    p = fma(p, z, cosf ? CL_COS_T12 : CL_SIN_T13);
    p = fma(p, z, cosf ? CL_COS_T10 : CL_SIN_T11);
    p = fma(p, z, cosf ? CL_COS_T8 : CL_SIN_T9);
    p = fma(p, z, cosf ? CL_COS_T6 : CL_SIN_T7);
    p = fma(p, z, cosf ? CL_COS_T4 : CL_SIN_T5);
    p = fma(p, z, cosf ? CL_COS_T2 : CL_SIN_T3);
    return cosf ? fma(z, p, 1.0) : fma(w.r * z, p, w.r);
}
// sin(x) bit-identical to cl_sincos's: quadrant 0 s, 1 c, 2 -s, 3 -c. Branch-free: a non-finite x reduces to a NaN
// r and gives NaN as cl_sincos does; x = +-0 reduces to r = +0, so the signed zero is selected.
__device__ __forceinline__ double cl_sin_split(const Reduced& w) {
    const double v = cl_poly(w, (w.q & 1) != 0);
    const double s = (w.q & 2) ? -v : v;
    return w.x == 0.0 ? w.x : s;
}
// cos(x) bit-identical to cl_sincos's: quadrant 0 c, 1 -s, 2 -c, 3 s (cos(+-0): r = +0, q = 0, exactly 1)
__device__ __forceinline__ double cl_cos_split(const Reduced& w) {
    const double v = cl_poly(w, (w.q & 1) == 0);
    return ((w.q + 1) & 2) ? -v : v;
}
// Float32 sin / cos from the same reduction: the hardware sine and cosine (special-function unit, absolute error
// below 2^-21.4 on [-pi, pi]) of the reduced argument |r| <= pi/4, then the quadrant. Two issue slots instead of
// two polynomials: the tangent's trigonometry is Float32 in the mixed kernels, and the orbit's stays Float64.
// Branch-free: quadrant 0 (s, c), 1 (c, -s), 2 (-s, -c), 3 (-c, s); a non-finite x has a NaN r, so NaN comes out.
__device__ __forceinline__ void cl_sincos32(const Reduced& w, float* sn, float* cs) {
    float s, c;
    __sincosf(static_cast<float>(w.r), &s, &c);
    const bool odd = (w.q & 1) != 0;
    const float a = odd ? c : s, b = odd ? s : c;
    *sn = (w.q & 2) ? -a : a;
    *cs = ((w.q + 1) & 2) ? -b : b;
}

__device__ __forceinline__ double cl_sin(double x) { double s, c; cl_sincos(x, &s, &c); return s; }
__device__ __forceinline__ double cl_cos(double x) { double s, c; cl_sincos(x, &s, &c); return c; }

__device__ __forceinline__ double cl_log(double x);

__device__ __forceinline__ double cl_log_impl(double x) {
    if (isnan(x)) return x;
    if (x < 0.0) return __longlong_as_double(0x7ff8000000000000LL);
    if (x == 0.0) return -__longlong_as_double(0x7ff0000000000000LL);
    if (isinf(x)) return x;
    double e = 0.0;
    unsigned long long b = static_cast<unsigned long long>(__double_as_longlong(x));
    if (x < 2.2250738585072014e-308) { b = static_cast<unsigned long long>(__double_as_longlong(x * 0x1p54)); e = -54.0; }
    e += static_cast<double>(static_cast<long long>((b >> 52) & 0x7ffULL) - 1023);
    double m = __longlong_as_double(static_cast<long long>((b & 0x000fffffffffffffULL) | 0x3ff0000000000000ULL));
    if (m > CL_SQRT2) { m = m * 0.5; e = e + 1.0; }
    const double f = m - 1.0;
    const double s = f / (2.0 + f);
    const double z = s * s;
    double R = CL_LOG_T9;
    R = fma(R, z, CL_LOG_T8);
    R = fma(R, z, CL_LOG_T7);
    R = fma(R, z, CL_LOG_T6);
    R = fma(R, z, CL_LOG_T5);
    R = fma(R, z, CL_LOG_T4);
    R = fma(R, z, CL_LOG_T3);
    R = fma(R, z, CL_LOG_T2);
    R = fma(R, z, CL_LOG_T1);
    R = R * z;
    const double hfsq = 0.5 * f * f;
    return e * CL_LN2_HI - ((hfsq - (s * (hfsq + R) + e * CL_LN2_LO)) - f);
}
__device__ __forceinline__ double cl_log(double x) { return cl_log_impl(x); }

// cl_exp: k = rint(x / ln 2), r = (x - k LN2_HI) - k LN2_LO (the first product exact), the Taylor polynomial of
// exp(r) to r^13 in Horner form, then the scaling by 2^k in at most two products (the first exact). Bitwise the
// oracle's p_exp.
__device__ __forceinline__ double cl_pow2(int k) { return __longlong_as_double(static_cast<long long>(k + 1023) << 52); }
__device__ __forceinline__ double cl_exp(double x) {
    if (isnan(x)) return x;
    if (x > 709.782712893384) return __longlong_as_double(0x7ff0000000000000LL);
    if (x < -745.1332191019412) return 0.0;
    const double k = rint(x * CL_INV_LN2);
    const double r = (x - k * CL_LN2_HI) - k * CL_LN2_LO;
    double p = CL_EXP_T13;
    p = fma(p, r, CL_EXP_T12);
    p = fma(p, r, CL_EXP_T11);
    p = fma(p, r, CL_EXP_T10);
    p = fma(p, r, CL_EXP_T9);
    p = fma(p, r, CL_EXP_T8);
    p = fma(p, r, CL_EXP_T7);
    p = fma(p, r, CL_EXP_T6);
    p = fma(p, r, CL_EXP_T5);
    p = fma(p, r, CL_EXP_T4);
    p = fma(p, r, CL_EXP_T3);
    p = fma(p, r, CL_EXP_T2);
    p = fma(p, r, 1.0);
    p = fma(p, r, 1.0);
    const int ki = static_cast<int>(k);
    if (ki > 1023) return (p * cl_pow2(1023)) * cl_pow2(ki - 1023);
    if (ki >= -1022) return p * cl_pow2(ki);
    return (p * cl_pow2(ki + 1000)) * cl_pow2(-1000);
}

// cl_atan2: the octant reduction to z = min / max in [0, 1]; atan(z) = atan(c) + atan(u), c = k / 16 the nearest
// table point, u = (z - c) / (1 + z c), |u| <= 1/32, atan(u) by its Taylor polynomial to u^13; then pi / 2 - a and
// pi - a with split constants, and the C99 special cases for zeros and infinities. Bitwise the oracle's p_atan2.
static __constant__ double c_atan_hi[17] = {CL_ATAN_HI_0, CL_ATAN_HI_1, CL_ATAN_HI_2, CL_ATAN_HI_3, CL_ATAN_HI_4,
    CL_ATAN_HI_5, CL_ATAN_HI_6, CL_ATAN_HI_7, CL_ATAN_HI_8, CL_ATAN_HI_9, CL_ATAN_HI_10, CL_ATAN_HI_11, CL_ATAN_HI_12,
    CL_ATAN_HI_13, CL_ATAN_HI_14, CL_ATAN_HI_15, CL_ATAN_HI_16};
static __constant__ double c_atan_lo[17] = {CL_ATAN_LO_0, CL_ATAN_LO_1, CL_ATAN_LO_2, CL_ATAN_LO_3, CL_ATAN_LO_4,
    CL_ATAN_LO_5, CL_ATAN_LO_6, CL_ATAN_LO_7, CL_ATAN_LO_8, CL_ATAN_LO_9, CL_ATAN_LO_10, CL_ATAN_LO_11, CL_ATAN_LO_12,
    CL_ATAN_LO_13, CL_ATAN_LO_14, CL_ATAN_LO_15, CL_ATAN_LO_16};
__device__ __forceinline__ double cl_atan01(double z) {
    const int k = static_cast<int>(rint(z * 16.0));
    const double c = k * 0.0625;
    const double u = (z - c) / (1.0 + z * c);
    const double u2 = u * u;
    double q = CL_ATAN_T13;
    q = fma(q, u2, CL_ATAN_T11);
    q = fma(q, u2, CL_ATAN_T9);
    q = fma(q, u2, CL_ATAN_T7);
    q = fma(q, u2, CL_ATAN_T5);
    q = fma(q, u2, CL_ATAN_T3);
    const double at = fma(u * u2, q, u);
    return c_atan_hi[k] + (at + c_atan_lo[k]);
}
__device__ __forceinline__ double cl_atan2(double y, double x) {
    if (isnan(x) || isnan(y)) return x + y;
    if (isinf(y)) {
        const double a = isinf(x) ? (x > 0 ? CL_PIO2_1 * 0.5 : (CL_PI_HI - CL_PIO2_1 * 0.5) + CL_PI_LO) : CL_PIO2_1;
        return copysign(a, y);
    }
    if (isinf(x)) return copysign(x > 0 ? 0.0 : CL_PI_HI, y);
    if (y == 0.0) return signbit(x) ? copysign(CL_PI_HI, y) : y;
    if (x == 0.0) return copysign(CL_PIO2_1, y);
    const double ax = fabs(x), ay = fabs(y);
    const bool swap = ay > ax;
    double a = cl_atan01(swap ? ax / ay : ay / ax);
    if (swap) a = (CL_PIO2_1 - a) + CL_PIO2_2;
    if (x < 0.0) a = (CL_PI_HI - a) + CL_PI_LO;
    return y < 0.0 ? -a : a;
}

// Neumaier compensated sum (src/Foundation/Foundation.jl:48-68); always Float64.
struct CS { double s, c; };
__device__ __forceinline__ void cs_add(CS& a, double y) {
    const double t = a.s + y;
    const double c = fabs(a.s) >= fabs(y) ? (a.s - t) + y : (y - t) + a.s;
    a.s = t;
    a.c = a.c + c;
}
__device__ __forceinline__ double cs_total(const CS& a) { return a.s + a.c; }

// safe_norm (src/Foundation/norm.jl:8-12) of a contiguous vector of N entries with stride 1, left folds.
template <int N, typename T>
__device__ __forceinline__ T safe_norm(const T* v) {
    T m = fabs(v[0]);
#pragma unroll
    for (int i = 1; i < N; ++i) m = jl_max(m, static_cast<T>(fabs(v[i])));
    if (!(isfin(m) && m > T(0))) return m;
    T q = v[0] / m;
    T s = q * q;
#pragma unroll
    for (int i = 1; i < N; ++i) { q = v[i] / m; s = s + q * q; }
    return m * sqrt(s);
}

// Norm, division and maximum of the reducers and the QR family. Float64: the reference's safe_norm, IEEE division
// and Julia's NaN-propagating max, so the plain kernels stay operation-for-operation. Float32 (mixed kernels): the
// unscaled norm sqrt(sum v^2) by the hardware reciprocal square root when the sum is a normal float (the scaled
// safe_norm otherwise), the fast reciprocal division (2 ulp) and fmaxf; the frames are renormalised every handoff, so their entries stay far inside the
// float range, and non-finite values are caught by the status check before any reducer runs.
template <int N, typename T>
__device__ __forceinline__ T nrm(const T* v) {
    if constexpr (sizeof(T) == 8) {
        return safe_norm<N>(v);
    } else {
        float s = v[0] * v[0];
#pragma unroll
        for (int i = 1; i < N; ++i) s = __fmaf_rn(v[i], v[i], s);
        if (s >= 1e-30f && s <= 1e30f) return s * rsqrtf(s);   // hardware reciprocal square root (2 ulp)
        return safe_norm<N>(v);
    }
}
// Square root: IEEE in Float64; in Float32 the hardware reciprocal square root for positive finite x.
template <typename T>
__device__ __forceinline__ T sqt(T x) {
    if constexpr (sizeof(T) == 8) {
        return sqrt(x);
    } else {
        return (x > 0.0f && x < __int_as_float(0x7f800000)) ? x * rsqrtf(x) : sqrtf(x);
    }
}
template <typename T>
__device__ __forceinline__ T dv(T a, T b) {
    if constexpr (sizeof(T) == 8) return a / b;
    else return __fdividef(a, b);
}
template <typename T>
__device__ __forceinline__ T mx(T a, T b) {
    if constexpr (sizeof(T) == 8) return jl_max(a, b);
    else return fmaxf(a, b);
}

// The logarithm of a norm or pivot, summed in Float64 either way: cl_log for the plain kernels; for the mixed
// kernels the hardware log2 of the Float32 value (relative error ~2^-22) times ln 2 in Float64.
template <typename T>
__device__ __forceinline__ double lnr(T a) {
    if constexpr (sizeof(T) == 8) return cl_log(a);
    else return static_cast<double>(__log2f(a)) * 0.6931471805599453;
}

// The element-type constants of the tolerances.
template <typename T> struct Eps;
template <> struct Eps<double> {
    static __device__ __forceinline__ double eps() { return 0x1p-52; }
    static __device__ __forceinline__ double floatmin() { return 2.2250738585072014e-308; }
};
template <> struct Eps<float> {
    static __device__ __forceinline__ float eps() { return 0x1p-23f; }
    static __device__ __forceinline__ float floatmin() { return 1.17549435e-38f; }
};

// splitmix64 finalizer `_mix` (src/Tangent/initial.jl:2-7), bitwise.
__device__ __forceinline__ uint64_t mix64(uint64_t z) {
    z += 0x9e3779b97f4a7c15ULL;
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
    return z ^ (z >> 31);
}

}  // namespace cl
