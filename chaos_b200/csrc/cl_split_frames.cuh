// cl_split_frames.cuh -- the split-precision orbit kernel of the coupled-maps ensemble: the orbit and the indicator
// frame in Float64, the Lyapunov frame in Float32.
//
// The path is the reference's `_orbit_body` (src/Tangent/orbit.jl:44-60) for FroeschleMap (froeschle_map.jl:9-58)
// carrying two frames along each orbit: QRSpectrum(HouseholderQR) with k = 4 (qr_spectrum.jl:50-73,
// householder.jl:19-80) and GALI_4 with SALI read off its columns 1-2 (gali.jl:156-169, sali.jl:98-111; a separate
// SALI run on the same orbit and W0 is bitwise GALI's columns 1-2, test/gali/ga_ac05_08.jl:356-397). Precision by
// what each output needs:
//   * the orbit: Float64, bit for bit the plain kernel's (the reference's own arithmetic), with sin and cos of the
//     three arguments from both Taylor polynomials of one reduction (cl_sincos, branch-free);
//   * the indicator frame (GALI, SALI): Float64. Its tangent entries a, b, c are the plain kernel's bit for bit; its
//     product exploits the tangent's structure ([[I, I], [A, I + A]]: 8 adds and 16 fmas per step instead of the
//     dense 64), and its handoff uses fused dots and hardware reciprocal square roots. Float32 does not hold these
//     indicators: on weakly chaotic orbits (lambda_1 ~ 1e-4 over 1e5 steps) the frame amplifies rounding by ~e^10,
//     which leaves Float32 SALI wrong by orders of magnitude and GALI_3, GALI_4 at the Float32 floor;
//   * the Lyapunov frame (QRSpectrum): Float32, a structure-exploiting Householder QR with fused dots (the diagonal
//     of R and the reflectors from the column norms, the reflectors applied only below and right of the pivot, Q
//     formed from the reflectors' nonzero blocks), which keeps the orthogonality loss near 4 eps(Float32), inside
//     the reference's threshold tol eps(T) k for every orbit;
//   * every logarithm of a norm or pivot: accumulated exactly as an exponent-tracked Float64 product per column
//     (m 2^e with m in [1, 2), one multiply and integer exponent arithmetic a handoff) and turned into the state's
//     compensated sum once, at the end of the launch: sum + comp = the same total to rounding of the logarithm.
//
// Layout: one orbit per thread, the point and both frames in registers, every reducer field the handoffs touch in
// this thread's slot of shared memory (the states are read once per handoff, so the registers hold only what every
// step needs). Only final records reach HBM, in the reference's state layouts (QRState, GALIState, SALIState).
#pragma once

#include "cl_kernel.cuh"

namespace cl {
namespace split {

// ---- arithmetic ---------------------------------------------------------------------------------------------------
// The reduction and polynomial constants of cl_sincos in constant memory: the multiply-adds read them as constant-bank
// operands, so the step loop keeps no register for them.
static __constant__ double c_red[4] = {CL_TWO_OVER_PI, CL_PIO2_1, CL_PIO2_2, CL_PIO2_3};
static __constant__ double c_sin[8] = {CL_SIN_T17, CL_SIN_T15, CL_SIN_T13, CL_SIN_T11, CL_SIN_T9, CL_SIN_T7, CL_SIN_T5,
                                       CL_SIN_T3};
static __constant__ double c_cos[8] = {CL_COS_T16, CL_COS_T14, CL_COS_T12, CL_COS_T10, CL_COS_T8, CL_COS_T6, CL_COS_T4,
                                       CL_COS_T2};

// cl_reduce with the constants from constant memory (the same operations in the same order)
__device__ __forceinline__ Reduced reduce_c(double x) {
    Reduced w;
    w.x = x;
    const double k = rint(x * c_red[0]);
    double r = fma(-k, c_red[1], x);
    r = fma(-k, c_red[2], r);
    r = fma(-k, c_red[3], r);
    w.r = r;
    w.z = r * r;
    w.q = static_cast<int>(static_cast<long long>(k) & 3);
    return w;
}

// sin(x) and cos(x) of a reduction, bit for bit cl_sincos's: both polynomials, then the quadrant by selects. A
// non-finite x gives NaN (its r is NaN); x = +-0 reduces to r = +0, so sin(x) = x is selected for the sign.
__device__ __forceinline__ void sincos_of(const Reduced& w, double* sn, double* cs) {
    const double z = w.z;
    double ps = c_sin[0];
#pragma unroll
    for (int i = 1; i < 8; ++i) ps = fma(ps, z, c_sin[i]);
    const double s = fma(w.r * z, ps, w.r);
    double pc = c_cos[0];
#pragma unroll
    for (int i = 1; i < 8; ++i) pc = fma(pc, z, c_cos[i]);
    const double c = fma(z, pc, 1.0);
    const bool odd = (w.q & 1) != 0;
    const double a = odd ? c : s, b = odd ? s : c;
    // the quadrant's signs as sign-bit flips: sin negative in quadrants 2, 3; cos in 1, 2
    const long long fs = static_cast<long long>(w.q & 2) << 62, fc = static_cast<long long>((w.q + 1) & 2) << 62;
    const double sv = __longlong_as_double(__double_as_longlong(a) ^ fs);
    *sn = (__double_as_longlong(w.x) << 1) == 0 ? w.x : sv;   // x = +-0, tested on the bits (the ALU, not the FP64 pipe)
    *cs = __longlong_as_double(__double_as_longlong(b) ^ fc);
}

// A positive running product m 2^e, m in [1, 2): multiply, then move the exponent into e (integer arithmetic). The
// factor is finite and positive (the handoffs check it first), so m a never under- or overflows.
struct LogProd { double m; int e; int pad; };
__device__ __forceinline__ void lp_mul(LogProd& p, double a) {
    const long long b = __double_as_longlong(p.m * a);
    p.e += static_cast<int>((b >> 52) & 0x7ff) - 1023;
    p.m = __longlong_as_double((b & 0x000fffffffffffffLL) | 0x3ff0000000000000LL);
}
// sum <- sum + log(m 2^e): e ln 2 in two exact-ish parts (e LN2_HI is exact for |e| < 2^20), then log m.
__device__ __forceinline__ void lp_flush(CS& sum, const LogProd& p) {
    const double e = static_cast<double>(p.e);
    cs_add(sum, e * CL_LN2_HI);
    cs_add(sum, fma(e, CL_LN2_LO, cl_log(p.m)));
}

// Float64 1 / sqrt(s) for a positive normal s (CUDA's rsqrt: a hardware estimate refined in Float64).
__device__ __forceinline__ double rsq64(double s) { return rsqrt(s); }

template <int N>
__device__ __forceinline__ float sumsq32(const float* v) {
    float s = v[0] * v[0];
#pragma unroll
    for (int i = 1; i < N; ++i) s = __fmaf_rn(v[i], v[i], s);
    return s;
}
template <int N>
__device__ __forceinline__ double sumsq64(const double* v) {
    double s = v[0] * v[0];
#pragma unroll
    for (int i = 1; i < N; ++i) s = fma(v[i], v[i], s);
    return s;
}
// max(|w|) over the frame is finite: every entry finite (the exact status check when a cheap one is inconclusive)
template <int N, typename T>
__device__ __forceinline__ bool finite_all(const T* w) {
    bool ok = true;
#pragma unroll
    for (int i = 0; i < N; ++i) ok = ok && isfin(w[i]);
    return ok;
}

// ---- the map ------------------------------------------------------------------------------------------------------
// FroeschleMap step at the old point (froeschle_map.jl:20-47): x' = x + p, the forward sines and cosine and the
// tangent's A = [[a, b], [b, c]] (_abc :35-39) bit for bit the plain kernel's, A rounded to Float32 for the Lyapunov
// frame.
struct Jac { double x1, x2, s1, s2, c12, a, b, c; float af, bf, cf; };

__device__ __forceinline__ void jac(double nu, double kappa, double mu, const double* z, Jac& J) {
    J.x1 = z[0] + z[2];
    J.x2 = z[1] + z[3];
    double c1, c2, s12;
    sincos_of(reduce_c(J.x1), &J.s1, &c1);
    sincos_of(reduce_c(J.x2), &J.s2, &c2);
    sincos_of(reduce_c(J.x1 + J.x2), &s12, &J.c12);
    const double t = mu * s12;
    J.a = -nu * c1 - t;
    J.b = -t;
    J.c = -kappa * c2 - t;
    J.af = static_cast<float>(J.a);
    J.bf = static_cast<float>(J.b);
    J.cf = static_cast<float>(J.c);
}
__device__ __forceinline__ void forward(double nu, double kappa, double mu, double* z, const Jac& J) {
    const double f = mu * (1.0 - J.c12);
    const double p1 = z[2] - nu * J.s1 - f;
    const double p2 = z[3] - kappa * J.s2 - f;
    z[0] = J.x1; z[1] = J.x2; z[2] = p1; z[3] = p2;
}
// W <- [[I, I], [A, I + A]] W, column by column: top = W_q + W_p, bottom = A top + W_p
template <int K>
__device__ __forceinline__ void apply32(const Jac& J, float* W) {
#pragma unroll
    for (int j = 0; j < K; ++j) {
        float* w = W + 4 * j;
        const float t1 = w[0] + w[2], t2 = w[1] + w[3];
        const float b1 = __fmaf_rn(J.af, t1, __fmaf_rn(J.bf, t2, w[2]));
        const float b2 = __fmaf_rn(J.bf, t1, __fmaf_rn(J.cf, t2, w[3]));
        w[0] = t1; w[1] = t2; w[2] = b1; w[3] = b2;
    }
}
template <int K>
__device__ __forceinline__ void apply64(const Jac& J, double* W) {
#pragma unroll
    for (int j = 0; j < K; ++j) {
        double* w = W + 4 * j;
        const double t1 = w[0] + w[2], t2 = w[1] + w[3];
        const double b1 = fma(J.a, t1, fma(J.b, t2, w[2]));
        const double b2 = fma(J.b, t1, fma(J.c, t2, w[3]));
        w[0] = t1; w[1] = t2; w[2] = b1; w[3] = b2;
    }
}

// ---- the Lyapunov frame: QRSpectrum(HouseholderQR), d = k = 4, Float32 -------------------------------------------
// The fields of QRState{Float64, 4} that the handoffs touch (the log sums live in `lp` until the end of the launch).
struct QRSlot {
    LogProd lp[4];
    double G_max, orth_max, value, threshold;
    i64 n, count_max, column, step;
    int code, pad;
};

// One handoff (qr_spectrum.jl:50-73 with householder.jl:19-80): W (4 x 4, column-major) is replaced by Q. The
// factorisation runs in W's own registers (A aliases W; its lower part is dead once the reflectors are taken, its
// upper part is R), so the handoff needs only the reflectors and R's inverse besides the frame.
__device__ __forceinline__ void qr_handoff(QRSlot& st, i64 n, float* W, double orth_tol) {
    float* A = W;
    float V[10], beta[3];   // reflector j: rows j..3 at V[off_j..], off = 0, 4, 7
    int count = 0;
#pragma unroll
    for (int j = 0; j < 3; ++j) {
        constexpr int off_tab[3] = {0, 4, 7};
        const int off = off_tab[j];
        float s2 = A[j + 4 * j] * A[j + 4 * j];
#pragma unroll
        for (int i = j + 1; i < 4; ++i) s2 = __fmaf_rn(A[i + 4 * j], A[i + 4 * j], s2);
        const float c = sqrtf(s2);
        float rho = c;
        beta[j] = 0.0f;
#pragma unroll
        for (int i = j; i < 4; ++i) V[off + i - j] = 0.0f;
        if (isfin(c) && c > 0.0f) {
            const float ajj = A[j + 4 * j];
            const float sg = ajj < 0.0f ? -1.0f : 1.0f;
            V[off] = ajj + sg * c;
#pragma unroll
            for (int i = j + 1; i < 4; ++i) V[off + i - j] = A[i + 4 * j];
            beta[j] = 1.0f / (c * (c + fabsf(ajj)));   // 2 / |v|^2
            // the columns right of the pivot, rows j..3: A_l -= beta (v . A_l) v
#pragma unroll
            for (int l = j + 1; l < 4; ++l) {
                float w = V[off] * A[j + 4 * l];
#pragma unroll
                for (int i = j + 1; i < 4; ++i) w = __fmaf_rn(V[off + i - j], A[i + 4 * l], w);
                const float f = beta[j] * w;
#pragma unroll
                for (int i = j; i < 4; ++i) A[i + 4 * l] = __fmaf_rn(-f, V[off + i - j], A[i + 4 * l]);
            }
            rho = -sg * c;
            count += 1;
        }
        A[j + 4 * j] = rho;
    }
    // _finish (householder.jl:66-75): R_ij = sg_i A_ij with sg_i the sign of A_ii, so that R_ii > 0
    float sg[4];
#pragma unroll
    for (int i = 0; i < 4; ++i) sg[i] = A[i + 4 * i] < 0.0f ? -1.0f : 1.0f;
#pragma unroll
    for (int j = 0; j < 4; ++j)
#pragma unroll
        for (int i = 0; i <= j; ++i) A[i + 4 * j] *= sg[i];
    int bad = 0;   // _factor_failure (qr_spectrum.jl:43-48): the first pivot that is not finite and positive
#pragma unroll
    for (int j = 3; j >= 0; --j)
        if (!(isfin(A[j + 4 * j]) && A[j + 4 * j] > 0.0f)) bad = j + 1;
    if (bad) {
        float pv = A[0];
#pragma unroll
        for (int j = 0; j < 4; ++j) if (j + 1 == bad) pv = A[j + 4 * j];
        st.code = 1; st.column = bad; st.value = pv; st.threshold = isfin(pv) ? 0.0 : __longlong_as_double(0x7ff0000000000000LL);
        st.step = n;
        return;
    }
    // window_Gw (orthonormalize.jl:112-127): |R|_F |R^-1|_F, R^-1 by back substitution with the pivots' reciprocals
    float rd[4], rin[4];
#pragma unroll
    for (int i = 0; i < 4; ++i) { rd[i] = A[i + 4 * i]; rin[i] = 1.0f / rd[i]; }
    float ra = 0.0f, rb = 0.0f;
    {
        float Ri[16];
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            Ri[j + 4 * j] = rin[j];
#pragma unroll
            for (int i = j - 1; i >= 0; --i) {
                float s = A[i + 4 * (i + 1)] * Ri[(i + 1) + 4 * j];
#pragma unroll
                for (int l = i + 2; l <= j; ++l) s = __fmaf_rn(A[i + 4 * l], Ri[l + 4 * j], s);
                Ri[i + 4 * j] = -s * rin[i];
            }
        }
#pragma unroll
        for (int j = 0; j < 4; ++j)
#pragma unroll
            for (int i = 0; i <= j; ++i) { ra = __fmaf_rn(A[i + 4 * j], A[i + 4 * j], ra); rb = __fmaf_rn(Ri[i + 4 * j], Ri[i + 4 * j], rb); }
    }
    const float Gw = sqrtf(ra) * sqrtf(rb);
    // Q = H_0 H_1 H_2 I, formed in W's registers (R is no longer needed but its diagonal, kept in rd): each H_j
    // touches rows j..3 of the columns j..3 (the columns left of j are still e_l there); then the column signs
    float* Q = W;
#pragma unroll
    for (int l = 0; l < 16; ++l) Q[l] = (l % 4) == (l / 4) ? 1.0f : 0.0f;
#pragma unroll
    for (int j = 2; j >= 0; --j) {
        constexpr int off_tab[3] = {0, 4, 7};
        const int off = off_tab[j];
#pragma unroll
        for (int l = j; l < 4; ++l) {
            float w = V[off] * Q[j + 4 * l];
#pragma unroll
            for (int i = j + 1; i < 4; ++i) w = __fmaf_rn(V[off + i - j], Q[i + 4 * l], w);
            const float f = beta[j] * w;
#pragma unroll
            for (int i = j; i < 4; ++i) Q[i + 4 * l] = __fmaf_rn(-f, V[off + i - j], Q[i + 4 * l]);
        }
    }
#pragma unroll
    for (int j = 0; j < 4; ++j)
#pragma unroll
        for (int i = 0; i < 4; ++i) Q[i + 4 * j] *= sg[j];
    // orth_loss (qr_spectrum.jl:4): max |Q'Q - I| over the upper triangle (Q'Q is symmetric)
    float orth = 0.0f;
#pragma unroll
    for (int j = 0; j < 4; ++j)
#pragma unroll
        for (int i = 0; i <= j; ++i) {
            float acc = Q[4 * i] * Q[4 * j];
#pragma unroll
            for (int q = 1; q < 4; ++q) acc = __fmaf_rn(Q[q + 4 * i], Q[q + 4 * j], acc);
            if (i == j) acc -= 1.0f;
            orth = fmaxf(orth, fabsf(acc));
        }
    const float thr = static_cast<float>(orth_tol) * 0x1p-23f * 4.0f;   // tol eps(Float32) k g, g = 1 (Householder)
    if (!(orth <= thr)) {
        st.code = 4; st.column = 0; st.value = orth; st.threshold = thr; st.step = n;
        return;
    }
#pragma unroll
    for (int i = 0; i < 4; ++i) lp_mul(st.lp[i], static_cast<double>(rd[i]));
    st.n = n;
    st.G_max = jl_max(st.G_max, static_cast<double>(Gw));   // _G_from_Gw is G_w for k > 2
    st.orth_max = jl_max(st.orth_max, static_cast<double>(orth));
    st.count_max = st.count_max > count ? st.count_max : count;
    st.column = 0;
}

// ---- the indicator frame: GALI_4 with SALI of its columns 1-2, Float64 ------------------------------------------
// `pending` marks a successful handoff whose values are not yet formed (bit 0: GALI's, bit 1: SALI's; below).
struct GSSlot {
    LogProd lp[4];
    double gali[3], gvalue, svalue, sali;
    i64 gn, gstep, gcolumn, sn, sstep;
    int gcode, scode, scolumn, pending;
};

// One handoff of the indicator frame without its values: the column norms, both reducers' failure checks, the log
// sums and the unit columns (which continue as the frame), as gali.jl:145-160 and sali.jl:100-110 run them. Of
// what a handoff writes only the stop decision and the frame depend on the norms alone; GALI's values (the nested
// Gram-Schmidt of the unit columns, gali.jl:156) and SALI's (min(d-, d+) of unit columns 1-2, sali.jl:108) are
// overwritten by every later successful handoff and read only after the last one. So they are formed once, by
// gali_values on the unit columns of the last successful handoff, bit for bit what forming them at every handoff
// leaves in the state. Returns whether the handoff succeeded (W then holds the unit columns).
__device__ __forceinline__ bool gali_step(GSSlot& st, i64 n, double* W) {
    double s[4], a[4], inv[4];
#pragma unroll
    for (int j = 0; j < 4; ++j) s[j] = sumsq64<4>(W + 4 * j);
    const double fm = 2.2250738585072014e-308;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        const bool pos = s[j] > 0.0 && isfin(s[j]);
        inv[j] = pos ? rsq64(s[j]) : 0.0;
        a[j] = pos ? s[j] * inv[j] : (s[j] == 0.0 ? 0.0 : safe_norm<4>(W + 4 * j));
        if (!pos && isfin(a[j]) && a[j] > 0.0) inv[j] = 1.0 / a[j];   // squares beyond the Float64 range
    }
    // SALI's own norm check on columns 1-2 (sali.jl:102-106), then GALI's (gali.jl:148-160: subnormal fails too)
    bool sali_ok = st.scode == 0;
    if (sali_ok) {
        const bool ok1 = isfin(a[0]) && a[0] > 0.0, ok2 = isfin(a[1]) && a[1] > 0.0;
        if (!(ok1 && ok2)) {
            st.scolumn = ok1 ? 2 : 1; st.svalue = ok1 ? a[1] : a[0]; st.sstep = n; st.scode = 1;
            sali_ok = false;
        }
    }
    int bad = 0;
#pragma unroll
    for (int j = 3; j >= 0; --j)
        if (!(isfin(a[j]) && a[j] >= fm)) bad = j + 1;
    if (bad) {
        double v = a[0];
#pragma unroll
        for (int j = 0; j < 4; ++j) if (j + 1 == bad) v = a[j];
        st.gvalue = v; st.gstep = n; st.gcode = 1; st.gcolumn = bad;
        return false;
    }
#pragma unroll
    for (int j = 0; j < 4; ++j) lp_mul(st.lp[j], a[j]);
#pragma unroll
    for (int j = 0; j < 4; ++j)
#pragma unroll
        for (int i = 0; i < 4; ++i) W[i + 4 * j] *= inv[j];
    if (sali_ok) st.sn = n;
    st.gn = n;
    st.pending = sali_ok ? 3 : 1;
    return true;
}

// The values of the last successful handoff from its unit columns U (column-major): SALI of columns 1-2 (sali.jl:
// 107-110) when that handoff ran SALI, and G_2..G_4 (gali.jl:81-100).
__device__ __forceinline__ void gali_values(GSSlot& st, const double* U) {
    if (st.pending & 2) {
        double dm = U[0] - U[4], dp = U[0] + U[4];
        double sm = dm * dm, sp = dp * dp;
#pragma unroll
        for (int i = 1; i < 4; ++i) {
            dm = U[i] - U[4 + i]; dp = U[i] + U[4 + i];
            sm = fma(dm, dm, sm); sp = fma(dp, dp, sp);
        }
        const double m = fmin(sm, sp);
        st.sali = m > 0.0 ? m * rsq64(m) : m;
    }
    double Q[16];
#pragma unroll
    for (int l = 0; l < 16; ++l) Q[l] = U[l];
    // _gram_core! (gali.jl:81-100): each column orthogonalised twice against the earlier (orthonormal) ones, then
    // normalised; G_k = prod_{i <= k} r_i. Each pass takes the projections on every earlier column at once (the
    // classical form, twice: the same orthogonality as the modified form for these few columns, with the dots
    // independent of one another)
    double g = 1.0;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
#pragma unroll
        for (int pass = 0; pass < 2; ++pass) {
            double cc[4];
#pragma unroll
            for (int p = 0; p < j; ++p) {
                cc[p] = Q[4 * p] * Q[4 * j];
#pragma unroll
                for (int i = 1; i < 4; ++i) cc[p] = fma(Q[i + 4 * p], Q[i + 4 * j], cc[p]);
            }
#pragma unroll
            for (int p = 0; p < j; ++p)
#pragma unroll
                for (int i = 0; i < 4; ++i) Q[i + 4 * j] = fma(-cc[p], Q[i + 4 * p], Q[i + 4 * j]);
        }
        const double r2 = sumsq64<4>(Q + 4 * j);
        const double ir = r2 > 0.0 ? rsq64(r2) : 1.0;
        const double r = r2 > 0.0 ? r2 * ir : 0.0;
#pragma unroll
        for (int i = 0; i < 4; ++i) Q[i + 4 * j] *= ir;
        if (j > 0) { g *= r; st.gali[j - 1] = g; }
    }
    st.pending = 0;
}

}  // namespace split
}  // namespace cl
