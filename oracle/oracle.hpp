// oracle/oracle.hpp -- TEST INFRASTRUCTURE (the CPU oracle). Only tests/, __graft_entry__.smoke() and the
// cpu_baseline / reference legs of bench.py use anything under oracle/; the product never does.
//
// A serial C++ restatement of Chaoslab's Float64 hot path, `propagate_orbit` (src/Tangent/orbit.jl:85-99) and the
// functions it calls, operation for operation: every product, sum and fma in the order the reference evaluates it
// (Julia contracts nothing; `fma` only where the reference writes it). Each function cites the reference lines it
// follows. Arithmetic that lives in third-party Julia packages is restated from their published definitions:
//  * StaticArrays.jl 1.9.23 -- `dot` and `sum`/`maximum` over an SVector are left folds of the plain products /
//    values (`_vecdot`, `_mapfoldl`); the SMatrix product `A * B` is the muladd chain of `fused_product`
//    (src/Foundation/product.jl:9-20 names it "the order of the StaticArrays product"), taken fused;
//  * LinearAlgebra `M \ B` on the 12 x 12 Gauss tangent system and `Matrix * Matrix`: reference LAPACK dgetf2 +
//    dgetrs (partial pivoting, first maximum) and reference BLAS dgemm order; Julia calls OpenBLAS there, whose
//    blocked order is not reproducible, so those bits are pinned only to rounding;
//  * Julia Base libm sin / cos / log: glibc (MATH_LIBM) or the portable functions of oracle_math.hpp.
// Parity of this restatement is pinned against the reference's own known-answer tests (closed forms and bitwise
// identities of test/tangent-core, test/lyap-*, test/megno, test/gali, test/coupled-maps, test/henon-heiles),
// which tests/ replay against it; the README value (StandardMap(6), lambda = 1.1348588476487835) is a sanity band
// because its seeded frame comes from StableRNGs.jl, which is absent.
#pragma once

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>

#include "../include/chaoslab_b200.h"
#include "oracle_math.hpp"

namespace orc {

constexpr double EPS = 0x1p-52;  // effective_eps(Float64) = eps(Float64), src/Foundation/Foundation.jl:44
constexpr double NaN = std::numeric_limits<double>::quiet_NaN();
constexpr double Inf = std::numeric_limits<double>::infinity();

// ---- Foundation ------------------------------------------------------------------------------------------------------
// Neumaier compensated sum, src/Foundation/Foundation.jl:48-68.
struct CS { double s, c; };
inline CS cs_add(CS a, double y) {
    const double t = a.s + y;
    const double c = std::fabs(a.s) >= std::fabs(y) ? (a.s - t) + y : (y - t) + a.s;
    return CS{t, a.c + c};
}
inline double cs_total(CS a) { return a.s + a.c; }

// safe_norm, src/Foundation/norm.jl:8-12: m = maximum(abs, v); m * sqrt(sum(abs2, v ./ m)), left folds.
inline double safe_norm(const double* v, int n) {
    double m = std::fabs(v[0]);
    for (int i = 1; i < n; ++i) m = jl_max(m, std::fabs(v[i]));
    if (!(isfin(m) && m > 0)) return m;
    double q = v[0] / m;
    double s = q * q;
    for (int i = 1; i < n; ++i) { q = v[i] / m; s = s + q * q; }
    return m * std::sqrt(s);
}

// fused_product, src/Foundation/product.jl:9-20: C[i,j] = A[i,1] B[1,j], then fma(A[i,q], B[q,j], acc), q ascending.
// A is m x p, B is p x n, all column-major.
inline void fused_product(const double* A, const double* B, double* C, int m, int p, int n) {
    for (int j = 0; j < n; ++j)
        for (int i = 0; i < m; ++i) {
            double acc = A[i] * B[j * p];
            for (int q = 1; q < p; ++q) acc = std::fma(A[i + q * m], B[q + j * p], acc);
            C[i + j * m] = acc;
        }
}

// ---- Julia-layout reducer states (T = Float64) ------------------------------------------------------------------
// Field order and alignment of the isbits structs; sizes are checked against Julia's sizeof below.
template <int K> struct QRStateJ {      // src/Lyapunov/qr_spectrum.jl:22-33
    CS sums[K]; int64_t n; double G_max, orth_max; int64_t count_max; int8_t code; int64_t column;
    double value, threshold; int64_t step;
};
struct BenettinStateJ {                 // src/Lyapunov/benettin.jl:14-20
    CS sum; int64_t n; int8_t code; double value; int64_t step;
};
struct SALIStateJ {                     // src/Indicators/sali.jl:17-26
    CS s1, s2; double sali, value; int64_t n, step; int8_t code, column;
};
template <int K> struct GALIStateJ {    // src/Indicators/gali.jl:20-29 (M = K - 1)
    double s[K], c[K], gali[K - 1]; double value; int64_t n, step; int8_t code; int64_t column;
};
struct MegnoSumsJ { CS s, R1, R2, Q, Q2; };   // src/Indicators/megno.jl:35-41
struct MEGNOStateJ {                    // src/Indicators/megno.jl:46-55
    MegnoSumsJ c1, c2; double value; int64_t n, K, step; int8_t code, column;
};
struct FLIStateJ {                      // src/Indicators/fli.jl:33-46
    CS s1, s2; double f1, fB, value; int64_t n, step, step1, stepB; int8_t code, column, colB;
};
struct RLIStateJ {                      // src/Indicators/rli.jl:30-40
    CS sA, sB, Q; double value; int64_t n, K, step; int8_t code, column;
};
static_assert(sizeof(RLIStateJ) == 88, "RLIState layout");
static_assert(sizeof(QRStateJ<2>) == 16 * 2 + 72, "QRState layout");
static_assert(sizeof(BenettinStateJ) == 48, "BenettinState layout");
static_assert(sizeof(SALIStateJ) == 72, "SALIState layout");
static_assert(sizeof(GALIStateJ<4>) == 24 * 4 + 32, "GALIState layout");
static_assert(sizeof(MEGNOStateJ) == 200, "MEGNOState layout");
static_assert(sizeof(FLIStateJ) == 96, "FLIState layout");

inline int64_t state_bytes_of(const cl_reducer& r, int k) {
    switch (r.kind) {
        case CL_RED_QR: return 16 * k + 72;
        case CL_RED_BENETTIN: return 48;
        case CL_RED_SALI: return 72;
        case CL_RED_GALI: return 24 * k + 32;
        case CL_RED_MEGNO: return 200;
        case CL_RED_FLI: return 96;
        case CL_RED_RLI: return 88;
    }
    return 0;
}

// ---- Systems ----------------------------------------------------------------------------------------------------------
// pi in Float64 as `_pi` builds it (src/Systems/standard_map.jl:46): 3.141592653589793 + 1.2246467991473532e-16.
inline double jl_pi() { return 3.141592653589793 + 1.2246467991473532e-16; }

// _reduce, src/Systems/wrapped_standard_map.jl:15-28.
inline void wrap_reduce(double u, double tp, double* r_out, double* a_out) {
    double a = std::floor(u / tp);
    double r = u - tp * a;
    if (r < 0) { r += tp; a -= 1; }
    if (r >= tp) { r -= tp; a += 1; }
    *r_out = r; *a_out = a;
}

// One step of the map (tangent at the OLD point, then forward), src/Tangent/orbit.jl:49-52, for the maps whose
// tangent is a dense SMatrix. `M` receives the d x d tangent (column-major), x is advanced in place.
template <int MM>
struct Systems {
    using Mth = Math<MM>;
    // StandardMap: forward standard_map.jl:18-21, tangent _dt standard_map.jl:30-34 ([[1+c, 1], [c, 1]], c = K cos x).
    static void standard(double K, double* x, double* M) {
        const double c = K * Mth::cos(x[0]);
        M[0] = 1.0 + c; M[1] = c; M[2] = 1.0; M[3] = 1.0;
        const double p = x[1] + K * Mth::sin(x[0]);
        x[0] = x[0] + p; x[1] = p;
    }
    // WrappedStandardMap forward, wrapped_standard_map.jl:30-37 (_checked :23-28), tangent _dt at x.
    static void wrapped(double K, double* z, double* M) {
        const double c = K * Mth::cos(z[0]);
        M[0] = 1.0 + c; M[1] = c; M[2] = 1.0; M[3] = 1.0;
        const double tp = 2 * jl_pi();
        double p, a, x, b;
        wrap_reduce(z[1] + K * Mth::sin(z[0]), tp, &p, &a);
        const double n = z[3] + a;
        wrap_reduce(z[0] + p, tp, &x, &b);
        const double m = z[2] + n + b;
        const double lim = 0x1p53;   // maxintfloat(Float64)
        if (std::fabs(m) < lim && std::fabs(n) < lim) { z[0] = x; z[1] = p; z[2] = m; z[3] = n; }
        else { z[0] = z[1] = z[2] = z[3] = NaN; }
    }
    // FroeschleMap forward froeschle_map.jl:20-25, tangent _f3_tangent :35-47 at the new positions x' = x + p.
    static void froeschle(double nu, double kappa, double mu, double* z, double* M) {
        const double x1 = z[0] + z[2], x2 = z[1] + z[3];
        // _abc: t = mu sin(x1 + x2); a = -nu cos x1 - t, b = -t, c = -kappa cos x2 - t
        const double t = mu * Mth::sin(x1 + x2);
        const double a = -nu * Mth::cos(x1) - t, b = -t, c = -kappa * Mth::cos(x2) - t;
        const double o = 1.0, Z = 0.0;
        const double Mv[16] = {o, Z, a, b, Z, o, b, c, o, Z, o + a, b, Z, o, b, o + c};
        std::memcpy(M, Mv, sizeof Mv);
        // forward: f = mu (1 - cos(x1' + x2')) (_fcoup :18)
        const double f = mu * (1.0 - Mth::cos(x1 + x2));
        const double p1 = z[2] - nu * Mth::sin(x1) - f;
        const double p2 = z[3] - kappa * Mth::sin(x2) - f;
        z[0] = x1; z[1] = x2; z[2] = p1; z[3] = p2;
    }
    // WrappedFroeschleMap, froeschle_map.jl:60-126, state (x1, x2, p1, p2, c1..c4): tangent _f3_tangent at the
    // unreduced sums u = x + p (:108); forward (:84-92) reduces the new positions (counts b), evaluates the force at
    // them, reduces the new momenta (counts a); m' = m + n + b, n' = n + a; _checked8 (:69-73).
    static void wrapped_froeschle(double nu, double kappa, double mu, double* z, double* M) {
        const double u1 = z[0] + z[2], u2 = z[1] + z[3];
        const double t = mu * Mth::sin(u1 + u2);
        const double a = -nu * Mth::cos(u1) - t, b = -t, c = -kappa * Mth::cos(u2) - t;
        const double o = 1.0, Z = 0.0;
        const double Mv[16] = {o, Z, a, b, Z, o, b, c, o, Z, o + a, b, Z, o, b, o + c};
        std::memcpy(M, Mv, sizeof Mv);
        const double tp = 2 * jl_pi();
        double x1, b1, x2, b2, p1, a1, p2, a2;
        wrap_reduce(u1, tp, &x1, &b1);
        wrap_reduce(u2, tp, &x2, &b2);
        const double f = mu * (1.0 - Mth::cos(x1 + x2));
        wrap_reduce(z[2] - nu * Mth::sin(x1) - f, tp, &p1, &a1);
        wrap_reduce(z[3] - kappa * Mth::sin(x2) - f, tp, &p2, &a2);
        const double m1 = z[4] + z[6] + b1, m2 = z[5] + z[7] + b2, n1 = z[6] + a1, n2 = z[7] + a2;
        const double lim = 0x1p53;
        if (std::fabs(m1) < lim && std::fabs(m2) < lim && std::fabs(n1) < lim && std::fabs(n2) < lim) {
            z[0] = x1; z[1] = x2; z[2] = p1; z[3] = p2; z[4] = m1; z[5] = m2; z[6] = n1; z[7] = n2;
        } else {
            for (int i = 0; i < 8; ++i) z[i] = NaN;
        }
    }
    // LinearSymplecticMap, linear_symplectic.jl: forward A z (StaticArrays product, fused), tangent A.
    static void linear(const double* A, int d, double* z, double* M) {
        double zn[CL_MAX_DIM];
        for (int i = 0; i < d; ++i) {
            double acc = A[i] * z[0];
            for (int q = 1; q < d; ++q) acc = std::fma(A[i + q * d], z[q], acc);
            zn[i] = acc;
        }
        std::memcpy(M, A, sizeof(double) * d * d);
        std::memcpy(z, zn, sizeof(double) * d);
    }
};

// StandardMapChain with the banded ChainTangent (src/Systems/standard_map_chain.jl:141-171, chain_tangent.jl:
// 38-61 / :62-97): the product `ChainTangent * W` is not a fused_product (the band has its own method).
template <int MM>
struct Chain {
    using Mth = Math<MM>;
    int N; double K, eps; bool ring;
    int left(int j) const { return j > 0 ? j - 1 : (ring ? N - 1 : -1); }   // 0-based; -1 = none
    int right(int j) const { return j < N - 1 ? j + 1 : (ring ? 0 : -1); }
    // _force :164-170
    double force(const double* q, int j) const {
        const int kl = left(j), kr = right(j);
        double s = 0.0;
        if (kl >= 0) s = s + Mth::sin(q[j] - q[kl]);
        if (kr >= 0) s = s + Mth::sin(q[j] - q[kr]);
        return K * Mth::sin(q[j]) + eps * s;
    }
    // The band of G at the OLD positions (_chain_tangent, chain_tangent.jl:84-91): diagonal (K cos q_j + eps cos
    // left) + eps cos right, off-diagonals minus those cosines.
    void band(const double* z, double* g, double* gl, double* gr) const {
        for (int j = 0; j < N; ++j) {
            const int kl = left(j), kr = right(j);
            const double g0 = K * Mth::cos(z[j]);
            const double cl = kl >= 0 ? eps * Mth::cos(z[j] - z[kl]) : 0.0;
            const double cr = kr >= 0 ? eps * Mth::cos(z[j] - z[kr]) : 0.0;
            g[j] = (g0 + cl) + cr; gl[j] = -cl; gr[j] = -cr;
        }
    }
    // `ChainTangent * W` (chain_tangent.jl:62-78): GW = _band(W_q) (:42-51); top = (W_q + GW) + W_p, bottom = GW + W_p.
    void apply(const double* g, const double* gl, const double* gr, double* W, int k) const {
        const int d = 2 * N;
        double Wn[CL_MAX_DIM * CL_MAX_K];
        for (int col = 0; col < k; ++col) {
            const double* Wq = W + col * d;
            const double* Wp = Wq + N;
            for (int j = 0; j < N; ++j) {
                const int kl = left(j), kr = right(j);
                double v = g[j] * Wq[j];
                if (kl >= 0) v = v + gl[j] * Wq[kl];
                if (kr >= 0) v = v + gr[j] * Wq[kr];
                Wn[col * d + j] = (Wq[j] + v) + Wp[j];
                Wn[col * d + N + j] = v + Wp[j];
            }
        }
        std::memcpy(W, Wn, sizeof(double) * d * k);
    }
    // forward of the fixed-size state (standard_map_chain.jl, `forward(m, z::SVector)`): p_j' = p_j + F_j(q),
    // q_j' = q_j + p_j'.
    void forward(double* z) const {
        double p[CL_MAX_DIM / 2];
        for (int j = 0; j < N; ++j) p[j] = z[N + j] + force(z, j);
        for (int j = 0; j < N; ++j) { z[j] = z[j] + p[j]; z[N + j] = p[j]; }
    }
    // WrappedStandardMapChain forward (wrapped_standard_map_chain.jl:117-124), state (q, p, counts of q, counts
    // of p): p~ = p + F(q) reduced (counts a), n' = n + a; q~ = q + p' reduced (counts b), m' = m + n' + b;
    // _guard_counts (:101-107). The band is the chain's at the reduced positions (:135-137).
    void forward_wrapped(double* z) const {
        const double tp = 2 * jl_pi();
        double p[CL_MAX_DIM / 2], nn[CL_MAX_DIM / 2];
        for (int j = 0; j < N; ++j) {
            double a;
            wrap_reduce(z[N + j] + force(z, j), tp, &p[j], &a);
            nn[j] = z[3 * N + j] + a;
        }
        bool ok = true;
        for (int j = 0; j < N; ++j) {
            double q, b;
            wrap_reduce(z[j] + p[j], tp, &q, &b);
            const double m = z[2 * N + j] + nn[j] + b;
            z[j] = q; z[N + j] = p[j]; z[2 * N + j] = m; z[3 * N + j] = nn[j];
            ok = ok && std::fabs(m) < 0x1p53 && std::fabs(nn[j]) < 0x1p53;
        }
        if (!ok) for (int i = 0; i < 4 * N; ++i) z[i] = NaN;
    }
};

// ---- Henon-Heiles flow and the Gauss-Legendre 3-stage method -------------------------------------------------------
// vector_field (flow_core.jl:78) with the Henon-Heiles force (flow_models.jl:102): (p, -F(q)),
// F = (q1 + 2 q1 q2, q2 + q1^2 - q2^2).
inline void hh_vf(const double* z, double* f) {
    const double F1 = z[0] + 2 * z[0] * z[1];
    const double F2 = (z[1] + z[0] * z[0]) - z[1] * z[1];
    f[0] = z[2]; f[1] = z[3]; f[2] = -F1; f[3] = -F2;
}
// vector_field_jacobian (flow_core.jl:79-83) with force_jacobian (flow_models.jl:103): [[0, I], [-Hs, 0]],
// Hs = [[1 + 2 q2, 2 q1], [2 q1, 1 - 2 q2]]; column-major 4 x 4.
inline void hh_jac(const double* z, double* J) {
    const double h11 = 1 + 2 * z[1], h21 = 2 * z[0], h12 = 2 * z[0], h22 = 1 - 2 * z[1];
    const double Jv[16] = {0, 0, -h11, -h21, 0, 0, -h12, -h22, 1, 0, 0, 0, 0, 1, 0, 0};
    std::memcpy(J, Jv, sizeof Jv);
}

struct Gauss3 {
    double Ahi[3][3], Alo[3][3], bhi[3], blo[3];
    int maxiter; double tol;  // tol NaN: the relative bound
    Gauss3(int maxiter_, double tol_) : maxiter(maxiter_), tol(tol_) {
        const double ah[3][3] = {{CL_GAUSS3_AHI_00, CL_GAUSS3_AHI_01, CL_GAUSS3_AHI_02},
                                 {CL_GAUSS3_AHI_10, CL_GAUSS3_AHI_11, CL_GAUSS3_AHI_12},
                                 {CL_GAUSS3_AHI_20, CL_GAUSS3_AHI_21, CL_GAUSS3_AHI_22}};
        const double al[3][3] = {{CL_GAUSS3_ALO_00, CL_GAUSS3_ALO_01, CL_GAUSS3_ALO_02},
                                 {CL_GAUSS3_ALO_10, CL_GAUSS3_ALO_11, CL_GAUSS3_ALO_12},
                                 {CL_GAUSS3_ALO_20, CL_GAUSS3_ALO_21, CL_GAUSS3_ALO_22}};
        std::memcpy(Ahi, ah, sizeof ah); std::memcpy(Alo, al, sizeof al);
        const double bh[3] = {CL_GAUSS3_BHI_0, CL_GAUSS3_BHI_1, CL_GAUSS3_BHI_2};
        const double bl[3] = {CL_GAUSS3_BLO_0, CL_GAUSS3_BLO_1, CL_GAUSS3_BLO_2};
        std::memcpy(bhi, bh, sizeof bh); std::memcpy(blo, bl, sizeof bl);
    }
    // _dot_comp, gauss.jl:91-101, per component: s, c start at 0; for j, for w in (hi_j, lo_j):
    // p = w F_j, pe = fma(w, F_j, -p); (s, se) = twosum(s, p) (stepper.jl:50-53); c = c + (se + pe); return s + c.
    static void dot_comp(const double* wh, const double* wl, const double F[3][4], double* out) {
        for (int l = 0; l < 4; ++l) {
            double s = 0.0, c = 0.0;
            for (int j = 0; j < 3; ++j)
                for (int h = 0; h < 2; ++h) {
                    const double w = h == 0 ? wh[j] : wl[j];
                    const double p = w * F[j][l];
                    const double pe = std::fma(w, F[j][l], -p);
                    const double t = s + p;
                    const double bb = t - s;
                    const double se = (s - (t - bb)) + (p - bb);
                    s = t;
                    c = c + (se + pe);
                }
            out[l] = s + c;
        }
    }
    // _gauss_core, gauss.jl:122-141 (compensated form, e = 0). Returns ok; inc and the final stages Y.
    bool core(const double* z, double h, double* inc, double Y[3][4]) const {
        double f0[4]; hh_vf(z, f0);
        for (int i = 0; i < 3; ++i) {
            const double ci = h * ((Ahi[i][0] + Ahi[i][1]) + Ahi[i][2]);
            for (int l = 0; l < 4; ++l) Y[i][l] = z[l] + ci * f0[l];
        }
        double F[3][4];
        for (int i = 0; i < 3; ++i) for (int l = 0; l < 4; ++l) F[i][l] = f0[l];
        double delta = 0.0, prev = Inf; bool stopped = false; int k = 0;
        while (k < maxiter && !stopped) {
            k += 1;
            for (int i = 0; i < 3; ++i) hh_vf(Y[i], F[i]);
            double Yn[3][4];
            for (int i = 0; i < 3; ++i) {
                double ss[4]; dot_comp(Ahi[i], Alo[i], F, ss);
                for (int l = 0; l < 4; ++l) Yn[i][l] = z[l] + (0.0 + h * ss[l]);
            }
            // _max_diff: maximum over stages of maximum(abs, Yn_i - Y_i)
            double dm = 0.0;
            for (int i = 0; i < 3; ++i) {
                double m = std::fabs(Yn[i][0] - Y[i][0]);
                for (int l = 1; l < 4; ++l) m = jl_max(m, std::fabs(Yn[i][l] - Y[i][l]));
                dm = i == 0 ? m : jl_max(dm, m);
            }
            delta = dm;
            std::memcpy(Y, Yn, sizeof Yn);
            if (!isfin(delta)) break;
            stopped = (delta == 0.0) || (k >= 2 && delta >= prev);
            prev = delta;
        }
        double bound;
        if (std::isnan(tol)) {
            double mn = 0.0;
            for (int i = 0; i < 3; ++i) {
                double m = std::fabs(Y[i][0]);
                for (int l = 1; l < 4; ++l) m = jl_max(m, std::fabs(Y[i][l]));
                mn = i == 0 ? m : jl_max(mn, m);
            }
            bound = 8 * EPS * jl_max(1.0, mn);
        } else {
            bound = tol;
        }
        const bool ok = stopped && isfin(delta) && delta <= bound;
        double us[4]; dot_comp(bhi, blo, F, us);
        for (int l = 0; l < 4; ++l) inc[l] = h * us[l];
        return ok;
    }
    // tangent_advance with W = I (gauss.jl:176-192 via IntegratorMap.tangent, integrator_map.jl:21) and the
    // advance it shares a core with (advance_n, gauss.jl:149-158, n = 1). M \ B: reference dgetf2 + dgetrs order;
    // Js[i] * dY_i: reference dgemm order (C = 0; for each l: C(:,j) += B(l,j) A(:,l)). Writes the 4 x 4 tangent T and advances z.
    void step(double* z, double h, double* T) const {
        double inc[4], Y[3][4];
        const bool ok = core(z, h, inc, Y);
        if (!ok) {
            for (int l = 0; l < 16; ++l) T[l] = NaN;   // W * NaN: every entry NaN
            for (int l = 0; l < 4; ++l) z[l] = NaN;
            return;
        }
        double J[3][16];
        for (int i = 0; i < 3; ++i) hh_jac(Y[i], J[i]);
        double A[3][3];
        for (int i = 0; i < 3; ++i) for (int j = 0; j < 3; ++j) A[i][j] = Ahi[i][j] + Alo[i][j];
        double M[12 * 12];   // column-major
        for (int c = 0; c < 12; ++c) for (int r = 0; r < 12; ++r) M[r + 12 * c] = r == c ? 1.0 : 0.0;
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j) {
                const double f = h * A[i][j];
                for (int c = 0; c < 4; ++c)
                    for (int r = 0; r < 4; ++r) {
                        double& e = M[(i * 4 + r) + 12 * (j * 4 + c)];
                        e = e - f * J[j][r + 4 * c];
                    }
            }
        double B[12 * 4];   // repeat(I, 3, 1)
        for (int c = 0; c < 4; ++c) for (int r = 0; r < 12; ++r) B[r + 12 * c] = (r % 4) == c ? 1.0 : 0.0;
        lu_solve12(M, B);
        double Wn[16];
        for (int l = 0; l < 16; ++l) Wn[l] = (l % 4) == (l / 4) ? 1.0 : 0.0;
        for (int i = 0; i < 3; ++i) {
            double P[16];
            // dgemm NN, beta = 0: C(:,j) = 0; for l: temp = B(l,j); C(i,j) = C(i,j) + temp * A(i,l)
            for (int jj = 0; jj < 4; ++jj) {
                for (int ii = 0; ii < 4; ++ii) P[ii + 4 * jj] = 0.0;
                for (int l = 0; l < 4; ++l) {
                    const double temp = B[(i * 4 + l) + 12 * jj];
                    for (int ii = 0; ii < 4; ++ii) P[ii + 4 * jj] = P[ii + 4 * jj] + temp * J[i][ii + 4 * l];
                }
            }
            const double f = h * (bhi[i] + blo[i]);
            for (int l = 0; l < 16; ++l) Wn[l] = Wn[l] + f * P[l];
        }
        std::memcpy(T, Wn, sizeof Wn);
        for (int l = 0; l < 4; ++l) z[l] = z[l] + inc[l];
    }
    // Unblocked right-looking LU with partial pivoting in the dgetf2 order (pivot = first index of the largest |a|,
    // column scaled by the reciprocal pivot, rank-1 update a(i,l) += a(i,j) * (-a(j,l)) skipped when a(j,l) = 0),
    // then the dgetrs solve: row swaps, unit-lower forward and upper backward substitution with the reference-BLAS
    // dtrsm zero skips. Julia runs OpenBLAS here; its blocked order is pinned only to rounding.
    static void lu_solve12(double* M, double* B) {
        int ipiv[12];
        for (int j = 0; j < 12; ++j) {
            int p = j; double pm = std::fabs(M[j + 12 * j]);
            for (int i = j + 1; i < 12; ++i) { const double a = std::fabs(M[i + 12 * j]); if (a > pm) { pm = a; p = i; } }
            ipiv[j] = p;
            if (M[p + 12 * j] != 0.0) {
                if (p != j) for (int c = 0; c < 12; ++c) std::swap(M[j + 12 * c], M[p + 12 * c]);
                const double rp = 1.0 / M[j + 12 * j];
                for (int i = j + 1; i < 12; ++i) M[i + 12 * j] = M[i + 12 * j] * rp;
            }
            for (int l = j + 1; l < 12; ++l) {
                const double t = -M[j + 12 * l];
                if (t != 0.0)
                    for (int i = j + 1; i < 12; ++i) M[i + 12 * l] = M[i + 12 * l] + M[i + 12 * j] * t;
            }
        }
        for (int j = 0; j < 12; ++j)
            if (ipiv[j] != j) for (int c = 0; c < 4; ++c) std::swap(B[j + 12 * c], B[ipiv[j] + 12 * c]);
        for (int c = 0; c < 4; ++c) {
            double* b = B + 12 * c;
            for (int k = 0; k < 12; ++k)
                if (b[k] != 0.0) for (int i = k + 1; i < 12; ++i) b[i] = b[i] - b[k] * M[i + 12 * k];
            for (int k = 11; k >= 0; --k)
                if (b[k] != 0.0) {
                    b[k] = b[k] / M[k + 12 * k];
                    for (int i = 0; i < k; ++i) b[i] = b[i] - b[k] * M[i + 12 * k];
                }
        }
    }
};

// ---- a table method on the Henon-Heiles flow: IntegratorMap(SplittingMethod(c, d), HenonHeilesFlow(), dt) ----
// force (flow_models.jl:102): (q1 + 2 q1 q2, q2 + q1^2 - q2^2), each as Julia evaluates it left to right.
inline void hh_force(double q1, double q2, double* F) {
    F[0] = q1 + (2 * q1) * q2;
    F[1] = (q2 + q1 * q1) - q2 * q2;
}
// drift (flow_core.jl:59): q += t p; kick (flow_core.jl:60): p -= t grad V(q).
inline void hh_drift(double* z, double t) { z[0] = z[0] + t * z[2]; z[1] = z[1] + t * z[3]; }
inline void hh_kick(double* z, double t) {
    double F[2];
    hh_force(z[0], z[1], F);
    z[2] = z[2] - t * F[0];
    z[3] = z[3] - t * F[1];
}
// drift_jacobian (flow_core.jl:64-67): [[I, t I], [0, I]], entries as built (t * 1, t * 0); column-major 4 x 4.
inline void hh_drift_jacobian(double t, double* J) {
    const double Jv[16] = {1, 0, 0, 0, 0, 1, 0, 0, t * 1.0, t * 0.0, 1, 0, t * 0.0, t * 1.0, 0, 1};
    std::memcpy(J, Jv, sizeof Jv);
}
// kick_jacobian (flow_core.jl:68-72) at the pre-kick point: [[I, 0], [-t Hs, I]], Hs = force_jacobian
// (flow_models.jl:103) = [[1 + 2 q2, 2 q1], [2 q1, 1 - 2 q2]], -t Hs formed as (-t) * Hs.
inline void hh_kick_jacobian(const double* z, double t, double* J) {
    const double h11 = 1 + 2 * z[1], h21 = 2 * z[0], h12 = 2 * z[0], h22 = 1 - 2 * z[1];
    const double mt = -t;
    const double Jv[16] = {1, 0, mt * h11, mt * h21, 0, 1, mt * h12, mt * h22, 0, 0, 1, 0, 0, 0, 0, 1};
    std::memcpy(J, Jv, sizeof Jv);
}

struct SplitHH {
    int n;
    const double* c;
    const double* d;
    int corr = 0;       // CorrectedMethod (stepper.jl:131-172): the corrector kick before and after each step
    double kap = 0.0;   // kappa = tau^3 eps^2 c / 2, eps = perturbation_scale(HenonHeilesFlow()) = 1
    static SplitHH of(const cl_system& s) {
        SplitHH m{s.n_stages, s.stage_c, s.stage_d};
        m.corr = s.corrector;
        m.kap = s.corrector ? (((s.dt * s.dt) * s.dt) * s.eps) / 2 : 0.0;
        return m;
    }
    // corrector_force (flow_models.jl:106): 2 (Hs g), the SMatrix-vector product a fused chain
    static void corrector_force(const double* z, double* C) {
        double f[4];
        hh_vf(z, f);   // (p, -F(q))
        const double F1 = -f[2], F2 = -f[3];
        const double h11 = 1 + 2 * z[1], h21 = 2 * z[0], h12 = 2 * z[0], h22 = 1 - 2 * z[1];
        C[0] = 2 * std::fma(h12, F2, h11 * F1);
        C[1] = 2 * std::fma(h22, F2, h21 * F1);
    }
    void corrector_kick(double* z) const {   // stepper.jl:136
        double C[2];
        corrector_force(z, C);
        z[2] = z[2] + kap * C[0];
        z[3] = z[3] + kap * C[1];
    }
    // _corrector_jacobian (stepper.jl:137-140) with corrector_hessian (flow_models.jl:107-112)
    void corrector_jacobian(const double* z, double* J) const {
        double f[4];
        hh_vf(z, f);
        const double F1 = -f[2], F2 = -f[3];
        const double h[4] = {1 + 2 * z[1], 2 * z[0], 2 * z[0], 1 - 2 * z[1]};
        const double t1[4] = {0, 2, 2, 0}, t2[4] = {2, 0, 0, -2};
        double hc[4];
        for (int j = 0; j < 2; ++j)
            for (int i = 0; i < 2; ++i) {
                const double hh = std::fma(h[i + 2], h[1 + 2 * j], h[i] * h[2 * j]);
                hc[i + 2 * j] = 2 * ((hh + F1 * t1[i + 2 * j]) + F2 * t2[i + 2 * j]);
            }
        const double Jv[16] = {1, 0, kap * hc[0], kap * hc[1], 0, 1, kap * hc[2], kap * hc[3], 0, 0, 1, 0, 0, 0, 0, 1};
        std::memcpy(J, Jv, sizeof Jv);
    }
    // tangent_advance with the identity frame (stepper.jl:108-118): per stage, drift then kick where the weight is
    // nonzero, each Jacobian (at the point before the sub-step) multiplied onto the frame by the StaticArrays
    // product (the fused chain of fused_product); the state advanced without merging kicks.
    void tangent(const double* x, double dt, double* T) const {
        double z[4] = {x[0], x[1], x[2], x[3]};
        double W[16] = {1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1}, J[16], Wn[16];
        if (corr) {
            corrector_jacobian(z, J);
            fused_product(J, W, Wn, 4, 4, 4);
            std::memcpy(W, Wn, sizeof W);
            corrector_kick(z);
        }
        for (int i = 0; i < n; ++i) {
            if (c[i] != 0.0) {
                const double t = c[i] * dt;
                hh_drift_jacobian(t, J);
                fused_product(J, W, Wn, 4, 4, 4);
                std::memcpy(W, Wn, sizeof W);
                hh_drift(z, t);
            }
            if (d[i] != 0.0) {
                const double t = d[i] * dt;
                hh_kick_jacobian(z, t, J);
                fused_product(J, W, Wn, 4, 4, 4);
                std::memcpy(W, Wn, sizeof W);
                hh_kick(z, t);
            }
        }
        if (corr) {
            corrector_jacobian(z, J);
            fused_product(J, W, Wn, 4, 4, 4);
            std::memcpy(W, Wn, sizeof W);
        }
        std::memcpy(T, W, sizeof W);
    }
    // advance_n(m, flow, z, dt, 1) (stepper.jl:27-48): kicks with no drift between them merged into one.
    void forward(double* z, double dt) const {
        if (corr) corrector_kick(z);
        double pend = 0.0;
        for (int i = 0; i < n; ++i) {
            const double ci = c[i];
            if (ci != 0.0) {
                if (pend != 0.0) { hh_kick(z, pend * dt); pend = 0.0; }
                hh_drift(z, ci * dt);
            }
            pend = pend + d[i];
        }
        if (pend != 0.0) hh_kick(z, pend * dt);
        if (corr) corrector_kick(z);
    }
    // the orbit body's map step: the tangent at the old point, then forward (orbit.jl:44-50)
    void step(double* x, double dt, double* T) const {
        tangent(x, dt, T);
        forward(x, dt);
    }
};

// ---- Orthonormalisers (src/Lyapunov/orthonormalize.jl, householder.jl) ---------------------------------------------
enum { QR_OK = 0, QR_PIVOT = 1, QR_PASSES = 2 };
constexpr int MAX_PASSES = 4;

inline double dotv(const double* a, const double* b, int n) {   // StaticArrays _vecdot: left fold of a_i b_i
    double s = a[0] * b[0];
    for (int i = 1; i < n; ++i) s = s + a[i] * b[i];
    return s;
}

struct QRResult { int count, status, column; };

// Gram-Schmidt family, orthonormalize.jl:38-105. W, Q: d x k; R: k x k (column-major).
inline QRResult orth_gs(int alg, const double* W, int d, int k, double* Q, double* R) {
    for (int l = 0; l < d * k; ++l) Q[l] = 0.0;
    for (int l = 0; l < k * k; ++l) R[l] = 0.0;
    QRResult res{1, QR_OK, 0};
    for (int m = 0; m < k; ++m) {
        const double* w = W + m * d;
        double u[CL_MAX_DIM] = {0}, r[CL_MAX_K] = {0};
        int passes = 1;
        for (int i = 0; i < d; ++i) u[i] = w[i];
        if (alg == CL_QR_CGS || alg == CL_QR_MGS) {          // :38-58
            for (int i = 0; i < m; ++i) {
                const double* qi = Q + i * d;
                const double c = dotv(qi, alg == CL_QR_CGS ? w : u, d);
                r[i] = c;
                for (int l = 0; l < d; ++l) u[l] = u[l] - c * qi[l];
            }
        } else {                                            // RGS :60-78
            const double eta = 1.0 / std::sqrt(2.0);
            double nold = safe_norm(w, d);
            passes = 0;
            for (;;) {
                passes += 1;
                double vold[CL_MAX_DIM];
                for (int l = 0; l < d; ++l) vold[l] = u[l];
                for (int i = 0; i < m; ++i) {
                    const double* qi = Q + i * d;
                    const double c = dotv(qi, vold, d);
                    r[i] = r[i] + c;
                    for (int l = 0; l < d; ++l) u[l] = u[l] - c * qi[l];
                }
                const double nnew = safe_norm(u, d);
                if (nnew >= nold * eta || !(isfin(nnew) && nnew > 0)) break;
                if (passes == MAX_PASSES) { passes = MAX_PASSES + 1; break; }
                nold = nnew;
            }
        }
        const double gamma = safe_norm(u, d);
        for (int i = 0; i < k; ++i) R[i + m * k] = i < m ? r[i] : (i == m ? gamma : 0.0);
        if (passes > MAX_PASSES) { res.status = QR_PASSES; res.column = m + 1; }
        else if (!(isfin(gamma) && gamma > 0)) { res.status = QR_PIVOT; res.column = m + 1; }
        if (res.status != QR_OK) break;
        for (int l = 0; l < d; ++l) Q[l + m * d] = u[l] / gamma;
        res.count = std::max(res.count, passes);
    }
    return res;
}

// _reflect (householder.jl:30-34): w_l = dot(u, A[:, l]); A = A - (2u) w'.  A is d x mcols.
inline void hh_reflect(double* A, const double* u, int d, int mcols) {
    double w[CL_MAX_K + CL_MAX_DIM];
    for (int l = 0; l < mcols; ++l) w[l] = dotv(u, A + l * d, d);
    for (int l = 0; l < mcols; ++l)
        for (int i = 0; i < d; ++i) A[i + l * d] = A[i + l * d] - (2 * u[i]) * w[l];
}
// _hh_sweep (householder.jl:37-50) with _reflector (:19-28); returns the count; U receives the reflectors.
inline int hh_sweep(double* A, int d, int mcols, int k, double* U) {
    const int nref = k < d ? k : k - 1;
    int count = 0;
    for (int l = 0; l < d * k; ++l) U[l] = 0.0;
    for (int j = 0; j < nref; ++j) {
        double a[CL_MAX_DIM] = {0};
        for (int i = 0; i < d; ++i) a[i] = i >= j ? A[i + j * d] : 0.0;
        const double c = safe_norm(a, d);
        double rho;
        if (isfin(c) && c > 0) {
            const double s = a[j] < 0 ? -1.0 : 1.0;
            a[j] = a[j] + s * c;
            const double nv = safe_norm(a, d);
            double u[CL_MAX_DIM];
            for (int i = 0; i < d; ++i) u[i] = a[i] / nv;
            rho = -s * c;
            hh_reflect(A, u, d, mcols);
            for (int i = 0; i < d; ++i) U[i + j * d] = u[i];
            count += 1;
        } else {
            rho = c;
        }
        A[j + j * d] = rho;
    }
    return count;
}
// _finish (householder.jl:66-75): sign fix and pivot status. Q d x k, A with leading dim ld.
inline QRResult hh_finish(double* Q, const double* A, int ld, int d, int k, int count, double* R) {
    double sg[CL_MAX_K];
    for (int j = 0; j < k; ++j) sg[j] = A[j + j * ld] < 0 ? -1.0 : 1.0;
    for (int j = 0; j < k; ++j)
        for (int i = 0; i < k; ++i) R[i + j * k] = i > j ? 0.0 : sg[i] * A[i + j * ld];
    for (int j = 0; j < k; ++j) for (int i = 0; i < d; ++i) Q[i + j * d] = Q[i + j * d] * sg[j];
    for (int j = 0; j < k; ++j) {
        const double p = R[j + j * k];
        if (!(isfin(p) && p > 0)) return QRResult{count, QR_PIVOT, j + 1};
    }
    return QRResult{count, QR_OK, 0};
}
inline QRResult orth_householder(const double* W, int d, int k, double* Q, double* R) {   // :77-80
    double A[CL_MAX_DIM * CL_MAX_K], U[CL_MAX_DIM * CL_MAX_K];
    std::memcpy(A, W, sizeof(double) * d * k);
    const int count = hh_sweep(A, d, k, k, U);
    // _form_q (:53-59): E = I[:, 1:k]; reflectors applied in reverse order
    for (int l = 0; l < d * k; ++l) Q[l] = (l % d) == (l / d) ? 1.0 : 0.0;
    const int nref = k < d ? k : k - 1;
    for (int j = nref - 1; j >= 0; --j) hh_reflect(Q, U + j * d, d, k);
    return hh_finish(Q, A, d, d, k, count, R);
}
inline QRResult orth_augmented(const double* W, int d, int k, double* Q, double* R) {     // :83-90
    double A[CL_MAX_DIM * (CL_MAX_K + CL_MAX_DIM)], U[CL_MAX_DIM * CL_MAX_K];
    const int mc = k + d;
    for (int l = 0; l < d * mc; ++l) {
        const int i = l % d, j = l / d;
        A[l] = l < d * k ? W[l] : (i == j - k ? 1.0 : 0.0);
    }
    const int count = hh_sweep(A, d, mc, k, U);
    for (int b = 0; b < k; ++b) for (int a = 0; a < d; ++a) Q[a + b * d] = A[b + (k + a) * d];   // _q_from_aug
    return hh_finish(Q, A, d, d, k, count, R);
}
// GivensQR (householder.jl:94-123): rows of [W, I_d]; rotations j = 1..min(k, d-1), i = d..j+1.
inline QRResult orth_givens(const double* W, int d, int k, double* Q, double* R) {
    const int wdt = k + d;
    double rows[CL_MAX_DIM][CL_MAX_K + CL_MAX_DIM];
    for (int i = 0; i < d; ++i)
        for (int l = 0; l < wdt; ++l) rows[i][l] = l < k ? W[i + l * d] : (l - k == i ? 1.0 : 0.0);
    int count = 0;
    const int J = std::min(k, d - 1);
    for (int j = 0; j < J; ++j)
        for (int i = d - 1; i >= j + 1; --i) {
            double* ra = rows[i - 1]; double* rb = rows[i];
            const double ab[2] = {ra[j], rb[j]};
            const double rho = safe_norm(ab, 2);
            if (!(isfin(rho) && rho > 0)) continue;
            const double c = ab[0] / rho, s = ab[1] / rho;
            double na[CL_MAX_K + CL_MAX_DIM], nb[CL_MAX_K + CL_MAX_DIM];
            for (int l = 0; l < wdt; ++l) { na[l] = c * ra[l] + s * rb[l]; nb[l] = c * rb[l] - s * ra[l]; }
            na[j] = rho; nb[j] = 0.0;
            std::memcpy(ra, na, sizeof(double) * wdt); std::memcpy(rb, nb, sizeof(double) * wdt);
            count += 1;
        }
    double R0[CL_MAX_K * CL_MAX_K];
    for (int j = 0; j < k; ++j) for (int i = 0; i < k; ++i) R0[i + j * k] = i > j ? 0.0 : rows[i][j];
    for (int b = 0; b < k; ++b) for (int a = 0; a < d; ++a) Q[a + b * d] = rows[b][k + a];
    return hh_finish(Q, R0, k, d, k, count, R);
}
inline QRResult orthonormalize(int alg, const double* W, int d, int k, double* Q, double* R) {
    switch (alg) {
        case CL_QR_CGS: case CL_QR_MGS: case CL_QR_RGS: return orth_gs(alg, W, d, k, Q, R);
        case CL_QR_HOUSEHOLDER: return orth_householder(W, d, k, Q, R);
        case CL_QR_AUGMENTED: return orth_augmented(W, d, k, Q, R);
        default: return orth_givens(W, d, k, Q, R);
    }
}

// window_Gw (orthonormalize.jl:112-127), k x k upper triangle.
inline double window_Gw(const double* R0, int k) {
    double R[CL_MAX_K * CL_MAX_K];
    std::memcpy(R, R0, sizeof(double) * k * k);
    double m = std::fabs(R[0]);
    for (int l = 1; l < k * k; ++l) m = jl_max(m, std::fabs(R[l]));
    if ((m > 1e100 || m < 1e-100) && isfin(m) && m > 0)
        for (int l = 0; l < k * k; ++l) R[l] = R[l] / m;
    double Ri[CL_MAX_K * CL_MAX_K] = {0};
    for (int j = 0; j < k; ++j) {
        Ri[j + j * k] = 1.0 / R[j + j * k];
        for (int i = j - 1; i >= 0; --i) {
            double s = 0.0;
            for (int l = i + 1; l <= j; ++l) s = s + R[i + l * k] * Ri[l + j * k];
            Ri[i + j * k] = -s / R[i + i * k];
        }
    }
    double a = R[0] * R[0], b = Ri[0] * Ri[0];
    for (int l = 1; l < k * k; ++l) { a = a + R[l] * R[l]; b = b + Ri[l] * Ri[l]; }
    return std::sqrt(a) * std::sqrt(b);
}
// _G_from_Gw (:130-132).
inline double G_from_Gw(double Gw, int k) {
    if (k == 1) return 1.0;
    if (k == 2) return (Gw + std::sqrt(jl_max(Gw * Gw - 4, 0.0))) / 2;
    return Gw;
}
// orth_loss (qr_spectrum.jl:4): maximum(abs, Q'Q - I), Q'Q as the fused StaticArrays product.
inline double orth_loss(const double* Q, int d, int k) {
    double m = 0.0; bool first = true;
    for (int j = 0; j < k; ++j)
        for (int i = 0; i < k; ++i) {
            double acc = Q[0 + i * d] * Q[0 + j * d];
            for (int q = 1; q < d; ++q) acc = std::fma(Q[q + i * d], Q[q + j * d], acc);
            if (i == j) acc = acc - 1.0;
            const double a = std::fabs(acc);
            m = first ? a : jl_max(m, a);
            first = false;
        }
    return m;
}

// ---- Reducers ---------------------------------------------------------------------------------------------------------
// Each step takes the state bytes, the global step n and W (d x k, replaced in place when the reducer replaces it),
// exactly as `reducer_step` (src/Tangent/Tangent.jl:44-49): never throws, records failures in the state.
template <int MM>
struct Reducers {
    using Mth = Math<MM>;

    // QRSpectrum, qr_spectrum.jl:50-73 (+ _factor_failure :43-48).
    static void qr(const cl_reducer& rd, uint8_t* st_bytes, int64_t n, double* W, int d, int k) {
        // QRState{Float64,K} with the runtime K: fields addressed by offsets of the Julia layout
        CS* sums = reinterpret_cast<CS*>(st_bytes);
        uint8_t* tail = st_bytes + 16 * k;
        int64_t* st_n = reinterpret_cast<int64_t*>(tail + 0);
        double* G_max = reinterpret_cast<double*>(tail + 8);
        double* orth_max = reinterpret_cast<double*>(tail + 16);
        int64_t* count_max = reinterpret_cast<int64_t*>(tail + 24);
        int8_t* code = reinterpret_cast<int8_t*>(tail + 32);
        int64_t* column = reinterpret_cast<int64_t*>(tail + 40);
        double* value = reinterpret_cast<double*>(tail + 48);
        double* threshold = reinterpret_cast<double*>(tail + 56);
        int64_t* step = reinterpret_cast<int64_t*>(tail + 64);
        if (*code != 0) return;
        double Q[CL_MAX_DIM * CL_MAX_K], R[CL_MAX_K * CL_MAX_K];
        const QRResult f = orthonormalize(rd.alg, W, d, k, Q, R);
        auto fail = [&](int c, int64_t col, double v, double thr) {
            *code = static_cast<int8_t>(c); *column = col; *value = v; *threshold = thr; *step = n;
        };
        if (f.status != QR_OK) {
            if (f.status == QR_PASSES) fail(2, f.column, MAX_PASSES + 1, MAX_PASSES);
            else {
                const double pv = R[(f.column - 1) + (f.column - 1) * k];
                fail(1, f.column, pv, isfin(pv) ? 0.0 : Inf);
            }
            return;
        }
        const double Gw = window_Gw(R, k);
        const bool gs = rd.alg == CL_QR_CGS || rd.alg == CL_QR_MGS || rd.alg == CL_QR_RGS;
        if (gs && !(Gw * EPS < 0.5)) { fail(3, 0, Gw * EPS, 0.5); return; }
        const double orth = k >= 2 ? orth_loss(Q, d, k) : 0.0;
        const double g = (rd.alg == CL_QR_CGS || rd.alg == CL_QR_MGS) ? Gw : 1.0;
        const double thr = rd.orthogonality_tol * EPS * static_cast<double>(k) * g;
        if (k >= 2 && !(orth <= thr)) { fail(4, 0, orth, thr); return; }
        for (int i = 0; i < k; ++i) sums[i] = cs_add(sums[i], Mth::log(R[i + i * k]));
        const double G = G_from_Gw(Gw, k);
        *st_n = n;
        *G_max = jl_max(*G_max, G);
        *orth_max = jl_max(*orth_max, orth);
        *count_max = std::max<int64_t>(*count_max, f.count);
        *column = 0;
        std::memcpy(W, Q, sizeof(double) * d * k);
    }

    // Benettin, benettin.jl:26-32.
    static void benettin(uint8_t* b, int64_t n, double* W, int d) {
        BenettinStateJ st; std::memcpy(&st, b, sizeof st);
        if (st.code != 0) return;
        const double alpha = safe_norm(W, d);
        if (!(isfin(alpha) && alpha > 0)) { st.code = 1; st.value = alpha; st.step = n; }
        else {
            st.sum = cs_add(st.sum, Mth::log(alpha)); st.n = n;
            for (int i = 0; i < d; ++i) W[i] = W[i] / alpha;
        }
        std::memcpy(b, &st, sizeof st);
    }

    // SALI, sali.jl:98-111 (unit_indices alignment.jl:11).
    static void sali(uint8_t* b, int64_t n, double* W, int d) {
        SALIStateJ st; std::memcpy(&st, b, sizeof st);
        if (st.code != 0) return;
        const double a1 = safe_norm(W, d), a2 = safe_norm(W + d, d);
        const bool ok1 = isfin(a1) && a1 > 0, ok2 = isfin(a2) && a2 > 0;
        if (!(ok1 && ok2)) {
            st.column = ok1 ? 2 : 1; st.value = ok1 ? a2 : a1; st.step = n; st.code = 1;
            std::memcpy(b, &st, sizeof st);
            return;
        }
        double u1[CL_MAX_DIM], u2[CL_MAX_DIM], dm[CL_MAX_DIM], dp[CL_MAX_DIM];
        for (int i = 0; i < d; ++i) { u1[i] = W[i] / a1; u2[i] = W[d + i] / a2; }
        for (int i = 0; i < d; ++i) { dm[i] = u1[i] - u2[i]; dp[i] = u1[i] + u2[i]; }
        st.s1 = cs_add(st.s1, Mth::log(a1));
        st.s2 = cs_add(st.s2, Mth::log(a2));
        st.sali = jl_min(safe_norm(dm, d), safe_norm(dp, d));
        st.n = n;
        for (int i = 0; i < d; ++i) { W[i] = u1[i]; W[d + i] = u2[i]; }
        std::memcpy(b, &st, sizeof st);
    }

    // _norm_col (gali.jl:47-58): the loop form of safe_norm over column j.
    static double norm_col(const double* c, int d) { return safe_norm(c, d); }

    // GALI, gali.jl:156-169 with _gram_core! (:81-100). GALIState{Float64, d, K, K-1} at runtime K.
    static void gali(uint8_t* b, int64_t n, double* W, int d, int K) {
        double* s = reinterpret_cast<double*>(b);
        double* c = s + K;
        double* gv = c + K;
        uint8_t* tail = b + 8 * (3 * K - 1);
        double* value = reinterpret_cast<double*>(tail);
        int64_t* st_n = reinterpret_cast<int64_t*>(tail + 8);
        int64_t* step = reinterpret_cast<int64_t*>(tail + 16);
        int8_t* code = reinterpret_cast<int8_t*>(tail + 24);
        int64_t* column = reinterpret_cast<int64_t*>(tail + 32);
        if (*code != 0) return;
        double a[CL_MAX_K];
        for (int j = 0; j < K; ++j) a[j] = norm_col(W + j * d, d);
        const double fm = std::numeric_limits<double>::min();
        for (int j = 0; j < K; ++j)
            if (!(isfin(a[j]) && a[j] >= fm)) {
                *value = a[j]; *step = n; *code = 1; *column = j + 1;
                return;
            }
        for (int j = 0; j < K; ++j) {
            const CS r = cs_add(CS{s[j], c[j]}, Mth::log(a[j]));
            s[j] = r.s; c[j] = r.c;
        }
        double Q[CL_MAX_DIM * CL_MAX_K];
        for (int j = 0; j < K; ++j) for (int i = 0; i < d; ++i) Q[i + j * d] = W[i + j * d] / a[j];
        std::memcpy(W, Q, sizeof(double) * d * K);   // W <- unit columns (before the nested QR)
        double g = 1.0;
        for (int j = 0; j < K; ++j) {
            double* qj = Q + j * d;
            for (int pass = 0; pass < 2; ++pass)
                for (int p = 0; p < j; ++p) {
                    const double* qp = Q + p * d;
                    double cc = 0.0;
                    for (int i = 0; i < d; ++i) cc = cc + qp[i] * qj[i];
                    for (int i = 0; i < d; ++i) qj[i] = qj[i] - cc * qp[i];
                }
            const double r = norm_col(qj, d);
            const double sc = r == 0.0 ? 1.0 : r;
            for (int i = 0; i < d; ++i) qj[i] = qj[i] / sc;
            if (j > 0) { g = g * r; gv[j - 1] = g; }
        }
        *st_n = n;
    }

    // MEGNO, megno.jl:63-80.
    static MegnoSumsJ megno_add(const MegnoSumsJ& m, double a, int64_t n) {
        const double tn = static_cast<double>(n);
        const CS R1 = cs_add(m.R1, tn * a), R2 = cs_add(m.R2, tn * tn * a);
        MegnoSumsJ o;
        o.s = cs_add(m.s, a); o.R1 = R1; o.R2 = R2;
        o.Q = cs_add(m.Q, 2 * cs_total(R1) / tn);
        o.Q2 = cs_add(m.Q2, 3 * cs_total(R2));
        return o;
    }
    static void megno(const cl_reducer& rd, uint8_t* b, int64_t n, double* W, int d) {
        MEGNOStateJ st; std::memcpy(&st, b, sizeof st);
        if (st.code != 0) return;
        const double a1 = safe_norm(W, d), a2 = safe_norm(W + d, d);
        const bool ok1 = isfin(a1) && a1 > 0, ok2 = isfin(a2) && a2 > 0;
        if (!(ok1 && ok2)) {
            st.column = ok1 ? 2 : 1; st.value = ok1 ? a2 : a1; st.step = n; st.code = 1;
            std::memcpy(b, &st, sizeof st);
            return;
        }
        const double l1 = Mth::log(a1), l2 = Mth::log(a2);
        st.c1 = megno_add(st.c1, l1, n);
        st.c2 = megno_add(st.c2, l2, n);
        st.n = n; st.K = st.K + 1;
        if (rd.replace) for (int i = 0; i < d; ++i) { W[i] = W[i] / a1; W[d + i] = W[d + i] / a2; }
        std::memcpy(b, &st, sizeof st);
    }

    // FLI, fli.jl:54-76.
    static void fli(const cl_reducer& rd, uint8_t* b, int64_t n, double* W, int d) {
        FLIStateJ st; std::memcpy(&st, b, sizeof st);
        if (st.code != 0) return;
        const double a1 = safe_norm(W, d), a2 = safe_norm(W + d, d);
        const bool ok1 = isfin(a1) && a1 > 0, ok2 = isfin(a2) && a2 > 0;
        if (!(ok1 && ok2)) {
            st.column = ok1 ? 2 : 1; st.value = ok1 ? a2 : a1; st.step = n; st.code = 1;
            std::memcpy(b, &st, sizeof st);
            return;
        }
        const CS s1 = cs_add(st.s1, Mth::log(a1)), s2 = cs_add(st.s2, Mth::log(a2));
        const double S1 = cs_total(s1), S2 = cs_total(s2);
        double f1 = st.f1; int64_t step1 = st.step1;
        if (S1 > st.f1) { f1 = S1; step1 = n; }
        double fB = st.fB; int64_t stepB = st.stepB; int8_t colB = st.colB;
        if (S1 > st.fB) { fB = S1; stepB = n; colB = 1; }
        if (S2 > fB) { fB = S2; stepB = n; colB = 2; }
        st.s1 = s1; st.s2 = s2; st.f1 = f1; st.fB = fB; st.n = n; st.step1 = step1; st.stepB = stepB; st.colB = colB;
        if (rd.replace) for (int i = 0; i < d; ++i) { W[i] = W[i] / a1; W[d + i] = W[d + i] / a2; }
        std::memcpy(b, &st, sizeof st);
    }

    // RLI's reducer_step (rli.jl:67-84) on a pair stream, d = 2h rows: norms as Benettin's, then the off-block check,
    // then the log sums, DL = |(sB.s - sA.s) + (sB.c - sA.c)| / n into Q, and the replacement when `replace`.
    static void rli(const cl_reducer& rd, uint8_t* b, int64_t n, double* W, int d) {
        RLIStateJ st; std::memcpy(&st, b, sizeof st);
        if (st.code != 0) return;
        const double a1 = safe_norm(W, d), a2 = safe_norm(W + d, d);
        const bool ok1 = isfin(a1) && a1 > 0, ok2 = isfin(a2) && a2 > 0;
        if (!(ok1 && ok2)) {
            st.column = ok1 ? 2 : 1; st.value = ok1 ? a2 : a1; st.step = n; st.code = 1;
            std::memcpy(b, &st, sizeof st);
            return;
        }
        const int h = d / 2;
        double m1 = 0.0, m2 = 0.0;
        for (int i = 0; i < h; ++i) { m1 = jl_max(m1, std::fabs(W[h + i])); m2 = jl_max(m2, std::fabs(W[d + i])); }
        if (!(m1 == 0 && m2 == 0)) {
            st.column = m1 == 0 ? 2 : 1; st.value = m1 == 0 ? m2 : m1; st.step = n; st.code = 2;
            std::memcpy(b, &st, sizeof st);
            return;
        }
        st.sA = cs_add(st.sA, Mth::log(a1));
        st.sB = cs_add(st.sB, Mth::log(a2));
        st.Q = cs_add(st.Q, std::fabs((st.sB.s - st.sA.s) + (st.sB.c - st.sA.c)) / static_cast<double>(n));
        st.n = n;
        st.K = st.K + 1;
        if (rd.replace) for (int i = 0; i < d; ++i) { W[i] = W[i] / a1; W[d + i] = W[d + i] / a2; }
        std::memcpy(b, &st, sizeof st);
    }

    static bool failed(const cl_reducer& rd, const uint8_t* b, int k) {
        switch (rd.kind) {
            case CL_RED_QR: return *reinterpret_cast<const int8_t*>(b + 16 * k + 32) != 0;
            case CL_RED_BENETTIN: return reinterpret_cast<const BenettinStateJ*>(b)->code != 0;
            case CL_RED_SALI: return reinterpret_cast<const SALIStateJ*>(b)->code != 0;
            case CL_RED_GALI: return *reinterpret_cast<const int8_t*>(b + 8 * (3 * k - 1) + 24) != 0;
            case CL_RED_MEGNO: return reinterpret_cast<const MEGNOStateJ*>(b)->code != 0;
            case CL_RED_FLI: return reinterpret_cast<const FLIStateJ*>(b)->code != 0;
            case CL_RED_RLI: return reinterpret_cast<const RLIStateJ*>(b)->code != 0;
        }
        return false;
    }

    static void step(const cl_reducer& rd, uint8_t* b, int64_t n, double* W, int d, int k) {
        switch (rd.kind) {
            case CL_RED_QR: qr(rd, b, n, W, d, k); break;
            case CL_RED_BENETTIN: benettin(b, n, W, d); break;
            case CL_RED_SALI: sali(b, n, W, d); break;
            case CL_RED_GALI: gali(b, n, W, d, k); break;
            case CL_RED_MEGNO: megno(rd, b, n, W, d); break;
            case CL_RED_FLI: fli(rd, b, n, W, d); break;
            case CL_RED_RLI: rli(rd, b, n, W, d); break;
        }
    }
};

// reducer_init (all zero fields) is the zero byte pattern for every state above.

// ---- Seeded Haar frames (initial.jl:1-34 key derivation; the stream itself is this project's own) -----------------
// splitmix64 finalizer `_mix`, initial.jl:2-7, bitwise.
inline uint64_t mix64(uint64_t z) {
    z += 0x9e3779b97f4a7c15ULL;
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
    return z ^ (z >> 31);
}
// Normal variates by Box-Muller from the counter stream u_t = (mix64(key + t) >> 11 + 1/2) 2^-53 (not StableRNGs:
// seeded frames are a different, documented stream), then two Gram-Schmidt passes per column, first k columns.
template <int MM>
inline void seeded_frame(uint64_t seed, int64_t orbit, int d, int k, double* W) {
    using Mth = Math<MM>;
    const uint64_t key = mix64(mix64(seed) + static_cast<uint64_t>(orbit));
    double G[CL_MAX_DIM * CL_MAX_DIM];
    const int nn = d * d;
    for (int t = 0; t < nn; t += 2) {
        const double u1 = (static_cast<double>(mix64(key + static_cast<uint64_t>(t)) >> 11) + 0.5) * 0x1p-53;
        const double u2 = (static_cast<double>(mix64(key + static_cast<uint64_t>(t) + 1) >> 11) + 0.5) * 0x1p-53;
        const double r = std::sqrt(-2.0 * Mth::log(u1));
        double sn, cs; Mth::sincos((2 * 3.141592653589793) * u2, &sn, &cs);
        G[t] = r * cs;
        if (t + 1 < nn) G[t + 1] = r * sn;
    }
    for (int j = 0; j < k; ++j) {
        double* g = G + j * d;
        for (int pass = 0; pass < 2; ++pass)
            for (int i = 0; i < j; ++i) {
                const double c = dotv(G + i * d, g, d);
                for (int l = 0; l < d; ++l) g[l] = g[l] - c * G[l + i * d];
            }
        double s = g[0] * g[0];
        for (int l = 1; l < d; ++l) s = s + g[l] * g[l];
        const double nr = std::sqrt(s);
        for (int l = 0; l < d; ++l) g[l] = g[l] / nr;
    }
    std::memcpy(W, G, sizeof(double) * d * k);
}

}  // namespace orc
