// cl_systems.cuh -- the maps of the fixed menu as device functors (src/Systems, src/Integrators).
//
// The orbit body evaluates the tangent at the OLD point and then advances the point (src/Tangent/orbit.jl:49-52).
// Each system splits that step in three so one point can drive several tangent frames:
//   jac(x, J)        everything the step needs at the old point (one sincos per distinct argument: `forward`
//                    and `tangent` of the reference evaluate the same arguments, so sharing them changes no bit)
//   apply<K>(J, W)   W <- tangent * W: for Real = double `fused_product` (src/Foundation/product.jl:9-20) on the
//                    reference's dense tangent matrix, including its 0 and 1 entries, or the band product of
//                    `ChainTangent` (chain_tangent.jl:62-78); for Real = float the same product exploiting the
//                    matrix structure
//   forward(x, J)    the new point, Float64 in every kernel, operation for operation the reference's `forward`.
#pragma once

#include <type_traits>

#include "cl_math.cuh"
#include "cl_reducers.cuh"

namespace cl {

// pi in Float64 as `_pi` builds it (src/Systems/standard_map.jl:46): 3.141592653589793 + 1.2246467991473532e-16.
__device__ __forceinline__ double jl_pi() {
    const double hi = 3.141592653589793, lo = 1.2246467991473532e-16;
    return hi + lo;
}

// fused_product of a dense D x D tangent M (column-major) with the D x K frame W, in place.
template <int D, int K>
__device__ __forceinline__ void fused_dense(const double* M, double* W) {
    double Wn[D * K];
#pragma unroll
    for (int j = 0; j < K; ++j)
#pragma unroll
        for (int i = 0; i < D; ++i) {
            double acc = M[i] * W[j * D];
#pragma unroll
            for (int q = 1; q < D; ++q) acc = fma(M[i + q * D], W[q + j * D], acc);
            Wn[i + j * D] = acc;
        }
#pragma unroll
    for (int l = 0; l < D * K; ++l) W[l] = Wn[l];
}
template <int D, int K>
__device__ __forceinline__ void fused_dense(const double* M, float* W) {   // mixed kernels: Float32 dense product
    float Wn[D * K];
#pragma unroll
    for (int j = 0; j < K; ++j)
#pragma unroll
        for (int i = 0; i < D; ++i) {
            float acc = static_cast<float>(M[i]) * W[j * D];
#pragma unroll
            for (int q = 1; q < D; ++q) acc = __fmaf_rn(static_cast<float>(M[i + q * D]), W[q + j * D], acc);
            Wn[i + j * D] = acc;
        }
#pragma unroll
    for (int l = 0; l < D * K; ++l) W[l] = Wn[l];
}

template <int D, int K>
__device__ __forceinline__ void fused_dense(const float* M, float* W) {    // mixed kernels: a Float32 tangent
    float Wn[D * K];
#pragma unroll
    for (int j = 0; j < K; ++j)
#pragma unroll
        for (int i = 0; i < D; ++i) {
            float acc = M[i] * W[j * D];
#pragma unroll
            for (int q = 1; q < D; ++q) acc = __fmaf_rn(M[i + q * D], W[q + j * D], acc);
            Wn[i + j * D] = acc;
        }
#pragma unroll
    for (int l = 0; l < D * K; ++l) W[l] = Wn[l];
}

// ---- StandardMap (standard_map.jl:8-44) and WrappedStandardMap (wrapped_standard_map.jl:12-57) -----------------
struct StdJac { double s, c; };   // sin x, K cos x at the old x
struct StdJacF { double s; float c; };   // mixed kernels: sin x in Float64 (orbit), K cos x in Float32 (tangent)

struct SysStandard {
    static constexpr int D = 2, S = 2;
    using Jac = StdJac;
    template <typename R> using JacR = typename std::conditional<sizeof(R) == 8, StdJac, StdJacF>::type;
    double K;
    __device__ __forceinline__ void jac(const double* x, StdJac& J) const {
        double sn, cs; cl_sincos(x[0], &sn, &cs);
        J.s = sn; J.c = K * cs;
    }
    __device__ __forceinline__ void jac(const double* x, StdJacF& J) const {
        const Reduced w = cl_reduce(x[0]);
        J.s = cl_sin_split(w);
        float sf, cf;
        cl_sincos32(w, &sf, &cf);
        J.c = static_cast<float>(K) * cf;
    }
    template <int KK>
    __device__ __forceinline__ void apply(const StdJacF& J, float* W) const {
        const float c = J.c, opc = 1.0f + J.c;
#pragma unroll
        for (int j = 0; j < KK; ++j) {
            const float w0 = W[2 * j], w1 = W[2 * j + 1];
            W[2 * j] = __fmaf_rn(opc, w0, w1);
            W[2 * j + 1] = __fmaf_rn(c, w0, w1);
        }
    }
    // _dt: [[1 + c, 1], [c, 1]]
    template <int KK>
    __device__ __forceinline__ void apply(const StdJac& J, double* W) const {
        const double o = 1.0;
        const double M[4] = {o + J.c, J.c, o, o};
        fused_dense<2, KK>(M, W);
    }
    template <int KK>
    __device__ __forceinline__ void apply(const StdJac& J, float* W) const {
        const float c = static_cast<float>(J.c), opc = static_cast<float>(1.0 + J.c);
#pragma unroll
        for (int j = 0; j < KK; ++j) {
            const float w0 = W[2 * j], w1 = W[2 * j + 1];
            W[2 * j] = __fmaf_rn(opc, w0, w1);
            W[2 * j + 1] = __fmaf_rn(c, w0, w1);
        }
    }
    template <class JJ>
    __device__ __forceinline__ void forward(double* x, const JJ& J) const {
        const double p = x[1] + K * J.s;
        x[0] = x[0] + p;
        x[1] = p;
    }
};

// _reduce (wrapped_standard_map.jl:15-28). The count a = floor(u / tp) of the IEEE quotient is taken from
// q = u * RN(1 / tp) where that is provably the same: |q - u / tp| <= 2^-52 |q| and RN(u / tp) lies within half an
// ulp of u / tp, so when the fraction of q is more than 2^-50 |q| + 2^-52 away from 0 and 1 (the 2^-52 covers the
// rounding of the fraction itself), floor(q) = floor(RN(u / tp)). Otherwise -- near an integer, 0, |q| >= 2^51,
// NaN or Inf -- the division decides, as in the reference. The remainder and the guards are the reference's.
__device__ __forceinline__ void wrap_reduce(double u, double tp, double& r, double& a) {
    const double q = u * (1.0 / tp);
    const double k = floor(q);
    const double f = q - k;
    const double margin = fabs(q) * 0x1p-50 + 0x1p-52;
    a = (f > margin && f < 1.0 - margin) ? k : floor(u / tp);
    r = u - tp * a;
    if (r < 0) { r += tp; a -= 1; }
    if (r >= tp) { r -= tp; a += 1; }
}

struct SysWrapped : SysStandard {
    static constexpr int S = 4;
    // forward (wrapped_standard_map.jl:30-37) with _checked (:23-28)
    template <class JJ>
    __device__ __forceinline__ void forward(double* z, const JJ& J) const {
        const double tp = 2 * jl_pi();
        double p, a, x, b;
        wrap_reduce(z[1] + K * J.s, tp, p, a);
        const double n = z[3] + a;
        wrap_reduce(z[0] + p, tp, x, b);
        const double m = z[2] + n + b;
        const double lim = 0x1p53;
        if (fabs(m) < lim && fabs(n) < lim) { z[0] = x; z[1] = p; z[2] = m; z[3] = n; }
        else { const double nan = __longlong_as_double(0x7ff8000000000000LL); z[0] = z[1] = z[2] = z[3] = nan; }
    }
};

// ---- FroeschleMap (froeschle_map.jl:9-58) ---------------------------------------------------------------------
struct FroJac { double x1, x2, s1, s2, c12, a, b, c; };
struct FroJacF { double x1, x2, s1, s2, c12; float a, b, c; };   // mixed: Float64 orbit terms, Float32 A

struct SysFroeschle {
    static constexpr int D = 4, S = 4;
    using Jac = FroJac;
    template <typename R> using JacR = typename std::conditional<sizeof(R) == 8, FroJac, FroJacF>::type;
    double nu, kappa, mu;
    // mixed: sin x1', sin x2', cos(x1' + x2') in Float64 bit-identical to the plain kernel's (the orbit), the
    // tangent's cos x1', cos x2', sin(x1' + x2') in Float32 from the same reductions
    __device__ __forceinline__ void jac(const double* z, FroJacF& J) const {
        J.x1 = z[0] + z[2];
        J.x2 = z[1] + z[3];
        const Reduced w1 = cl_reduce(J.x1), w2 = cl_reduce(J.x2), w12 = cl_reduce(J.x1 + J.x2);
        J.s1 = cl_sin_split(w1);
        J.s2 = cl_sin_split(w2);
        J.c12 = cl_cos_split(w12);
        float s1f, c1f, s2f, c2f, s12f, c12f;
        cl_sincos32(w1, &s1f, &c1f);
        cl_sincos32(w2, &s2f, &c2f);
        cl_sincos32(w12, &s12f, &c12f);
        const float t = static_cast<float>(mu) * s12f;
        J.a = -static_cast<float>(nu) * c1f - t;
        J.b = -t;
        J.c = -static_cast<float>(kappa) * c2f - t;
    }
    __device__ __forceinline__ void jac(const double* z, FroJac& J) const {
        J.x1 = z[0] + z[2];
        J.x2 = z[1] + z[3];
        double c1, c2, s12;
        cl_sincos(J.x1, &J.s1, &c1);
        cl_sincos(J.x2, &J.s2, &c2);
        cl_sincos(J.x1 + J.x2, &s12, &J.c12);
        const double t = mu * s12;               // _abc (:35-39)
        J.a = -nu * c1 - t;
        J.b = -t;
        J.c = -kappa * c2 - t;
    }
    // M = [[I, I], [A, I + A]] (_f3_tangent :42-47), the dense fused product with every 0 and 1 entry
    template <int KK>
    __device__ __forceinline__ void apply(const FroJac& J, double* W) const {
        const double o = 1.0, Z = 0.0;
        const double M[16] = {o, Z, J.a, J.b, Z, o, J.b, J.c, o, Z, o + J.a, J.b, Z, o, J.b, o + J.c};
        fused_dense<4, KK>(M, W);
    }
    // Float32: top = W_q + W_p, bottom = A (W_q + W_p) + W_p
    template <int KK, class JJ>
    __device__ __forceinline__ void apply(const JJ& J, float* W) const {
        const float a = static_cast<float>(J.a), b = static_cast<float>(J.b), c = static_cast<float>(J.c);
#pragma unroll
        for (int j = 0; j < KK; ++j) {
            float* w = W + 4 * j;
            const float t1 = w[0] + w[2], t2 = w[1] + w[3];
            const float b1 = __fmaf_rn(a, t1, __fmaf_rn(b, t2, w[2]));
            const float b2 = __fmaf_rn(b, t1, __fmaf_rn(c, t2, w[3]));
            w[0] = t1; w[1] = t2; w[2] = b1; w[3] = b2;
        }
    }
    template <class JJ>
    __device__ __forceinline__ void forward(double* z, const JJ& J) const {   // :20-25
        const double f = mu * (1.0 - J.c12);
        const double p1 = z[2] - nu * J.s1 - f;
        const double p2 = z[3] - kappa * J.s2 - f;
        z[0] = J.x1; z[1] = J.x2; z[2] = p1; z[3] = p2;
    }
};

// ---- WrappedFroeschleMap (froeschle_map.jl:60-126) -----------------------------------------------------------------
// State (x1, x2, p1, p2, c1, c2, c3, c4). The tangent is _f3_tangent at the UNREDUCED sums u = x + p (:108), the
// forward map's sines at the reduced new positions (:84-92): six trigonometric arguments per step, not three.
struct WFroJac { double x1, x2, b1, b2, s1, s2, c12, a, b, c; };
struct WFroJacF { double x1, x2, b1, b2, s1, s2, c12; float a, b, c; };   // mixed: Float32 A

struct SysWrappedFroeschle {
    static constexpr int D = 4, S = 8;
    using Jac = WFroJac;
    template <typename R> using JacR = typename std::conditional<sizeof(R) == 8, WFroJac, WFroJacF>::type;
    double nu, kappa, mu;
    // positions reduced with their counts, then the forward map's Float64 sines (split evaluation, bit-identical
    // to cl_sincos)
    template <class JJ>
    __device__ __forceinline__ void positions(double u1, double u2, JJ& J) const {
        const double tp = 2 * jl_pi();
        wrap_reduce(u1, tp, J.x1, J.b1);
        wrap_reduce(u2, tp, J.x2, J.b2);
        J.s1 = cl_sin_split(cl_reduce(J.x1));
        J.s2 = cl_sin_split(cl_reduce(J.x2));
        J.c12 = cl_cos_split(cl_reduce(J.x1 + J.x2));
    }
    __device__ __forceinline__ void jac(const double* z, WFroJac& J) const {
        const double u1 = z[0] + z[2], u2 = z[1] + z[3];
        const double t = mu * cl_sin_split(cl_reduce(u1 + u2));   // _abc (:35-39) at the unreduced sums
        J.a = -nu * cl_cos_split(cl_reduce(u1)) - t;
        J.b = -t;
        J.c = -kappa * cl_cos_split(cl_reduce(u2)) - t;
        positions(u1, u2, J);
    }
    __device__ __forceinline__ void jac(const double* z, WFroJacF& J) const {
        const double u1 = z[0] + z[2], u2 = z[1] + z[3];
        float s1f, c1f, s2f, c2f, s12f, c12f;
        cl_sincos32(cl_reduce(u1), &s1f, &c1f);
        cl_sincos32(cl_reduce(u2), &s2f, &c2f);
        cl_sincos32(cl_reduce(u1 + u2), &s12f, &c12f);
        const float t = static_cast<float>(mu) * s12f;
        J.a = -static_cast<float>(nu) * c1f - t;
        J.b = -t;
        J.c = -static_cast<float>(kappa) * c2f - t;
        positions(u1, u2, J);
    }
    template <int KK>
    __device__ __forceinline__ void apply(const WFroJac& J, double* W) const {   // the dense fused product
        const double o = 1.0, Z = 0.0;
        const double M[16] = {o, Z, J.a, J.b, Z, o, J.b, J.c, o, Z, o + J.a, J.b, Z, o, J.b, o + J.c};
        fused_dense<4, KK>(M, W);
    }
    template <int KK>
    __device__ __forceinline__ void apply(const WFroJacF& J, float* W) const {   // [[I, I], [A, I + A]] by blocks
#pragma unroll
        for (int j = 0; j < KK; ++j) {
            float* w = W + 4 * j;
            const float t1 = w[0] + w[2], t2 = w[1] + w[3];
            const float b1 = __fmaf_rn(J.a, t1, __fmaf_rn(J.b, t2, w[2]));
            const float b2 = __fmaf_rn(J.b, t1, __fmaf_rn(J.c, t2, w[3]));
            w[0] = t1; w[1] = t2; w[2] = b1; w[3] = b2;
        }
    }
    // forward (:84-92) with _checked8 (:69-73): momenta reduced with their counts, m' = m + n + b, n' = n + a
    template <class JJ>
    __device__ __forceinline__ void forward(double* z, const JJ& J) const {
        const double tp = 2 * jl_pi();
        const double f = mu * (1.0 - J.c12);
        double p1, a1, p2, a2;
        wrap_reduce(z[2] - nu * J.s1 - f, tp, p1, a1);
        wrap_reduce(z[3] - kappa * J.s2 - f, tp, p2, a2);
        const double m1 = z[4] + z[6] + J.b1, m2 = z[5] + z[7] + J.b2, n1 = z[6] + a1, n2 = z[7] + a2;
        const double lim = 0x1p53;
        if (fabs(m1) < lim && fabs(m2) < lim && fabs(n1) < lim && fabs(n2) < lim) {
            z[0] = J.x1; z[1] = J.x2; z[2] = p1; z[3] = p2; z[4] = m1; z[5] = m2; z[6] = n1; z[7] = n2;
        } else {
            const double nan = __longlong_as_double(0x7ff8000000000000LL);
#pragma unroll
            for (int i = 0; i < 8; ++i) z[i] = nan;
        }
    }
};

// ---- LinearSymplecticMap (linear_symplectic.jl): z' = A z (fused StaticArrays product), tangent A ----------------
template <int DD>
struct SysLinear {
    static constexpr int D = DD, S = DD;
    double A[D * D];   // the d x d matrix (column-major), passed by value: kernel-parameter (constant bank) loads
    struct Jac {};
    template <typename R> using JacR = Jac;
    __device__ __forceinline__ void jac(const double*, Jac&) const {}
    template <int KK, typename T>
    __device__ __forceinline__ void apply(const Jac&, T* W) const { fused_dense<D, KK>(A, W); }
    __device__ __forceinline__ void forward(double* z, const Jac&) const {
        double zn[D];
#pragma unroll
        for (int i = 0; i < D; ++i) {
            double acc = A[i] * z[0];
#pragma unroll
            for (int q = 1; q < D; ++q) acc = fma(A[i + q * D], z[q], acc);
            zn[i] = acc;
        }
#pragma unroll
        for (int i = 0; i < D; ++i) z[i] = zn[i];
    }
};

// ---- StandardMapChain with the banded ChainTangent (standard_map_chain.jl, chain_tangent.jl) -------------------
// Neighbours are compile-time per boundary (the ring flag is uniform over a launch, so the branch on it costs
// nothing and every index stays static, keeping the frame in registers). Each bond (j, j+1) is evaluated once:
// sin(q_j - q_j+1) = -sin(q_j+1 - q_j) and cos(q_j - q_j+1) = cos(q_j+1 - q_j) hold bitwise for the portable
// functions (the reduction and both polynomials are odd / even in the argument, and q_j+1 - q_j = -(q_j - q_j+1)
// exactly); the only difference, the sign of a zero sine, is erased by `_force`'s 0 + s (standard_map_chain.jl:166).
template <int NS>
struct ChainJac { double g[NS], gl[NS], gr[NS], sq[NS], sl[NS], sr[NS]; };
template <int NS>
struct ChainJacF { float g[NS], gl[NS], gr[NS]; double sq[NS], sl[NS], sr[NS]; };

template <int NS>
struct SysChain {
    static constexpr int D = 2 * NS, S = 2 * NS;
    using Jac = ChainJac<NS>;
    template <typename R> using JacR = typename std::conditional<sizeof(R) == 8, ChainJac<NS>, ChainJacF<NS>>::type;
    double K, eps;
    int ring;
    template <bool RING> static __device__ __forceinline__ constexpr int L(int j) { return j > 0 ? j - 1 : (RING ? NS - 1 : -1); }
    template <bool RING> static __device__ __forceinline__ constexpr int R(int j) { return j < NS - 1 ? j + 1 : (RING ? 0 : -1); }

    // _chain_tangent (chain_tangent.jl:84-91) at the old positions and the sines `_force` needs (:164-170).
    template <bool RING, class JJ>
    __device__ __forceinline__ void jac_impl(const double* z, JJ& J) const {
        constexpr bool F32 = sizeof(J.g[0]) == 4;
        double sb[NS], cb[NS];     // bond j: q_j - q_R(j), Float64 sine (orbit), cosine in the tangent's type
        float cbf[NS];
#pragma unroll
        for (int j = 0; j < NS; ++j) {
            if (R<RING>(j) < 0) continue;
            const double y = z[j] - z[R<RING>(j)];
            if constexpr (F32) {
                const Reduced w = cl_reduce(y);
                sb[j] = cl_sin_split(w);
                float sf; cl_sincos32(w, &sf, &cbf[j]);
                cb[j] = 0.0;
            } else {
                cl_sincos(y, &sb[j], &cb[j]);
                cbf[j] = 0.0f;
            }
        }
#pragma unroll
        for (int j = 0; j < NS; ++j) {
            const int kl = L<RING>(j), kr = R<RING>(j);
            double sq, cq = 0.0;
            float cqf = 0.0f;
            if constexpr (F32) {
                const Reduced w = cl_reduce(z[j]);
                sq = cl_sin_split(w);
                float sf; cl_sincos32(w, &sf, &cqf);
            } else {
                cl_sincos(z[j], &sq, &cq);
            }
            // left neighbour kl = j - 1 (or N - 1 for j = 0 on a ring): bond kl, sine negated
            const double sl = kl >= 0 ? -sb[kl] : 0.0;
            const double sr = kr >= 0 ? sb[j] : 0.0;
            J.sq[j] = sq; J.sl[j] = sl; J.sr[j] = sr;
            if constexpr (F32) {
                const float e = static_cast<float>(eps);
                const float cl_ = kl >= 0 ? e * cbf[kl] : 0.0f, cr = kr >= 0 ? e * cbf[j] : 0.0f;
                J.g[j] = (static_cast<float>(K) * cqf + cl_) + cr;
                J.gl[j] = -cl_;
                J.gr[j] = -cr;
            } else {
                const double cl_ = kl >= 0 ? eps * cb[kl] : 0.0, cr = kr >= 0 ? eps * cb[j] : 0.0;
                J.g[j] = (K * cq + cl_) + cr;
                J.gl[j] = -cl_;
                J.gr[j] = -cr;
            }
        }
    }
    template <class JJ>
    __device__ __forceinline__ void jac(const double* z, JJ& J) const {
        if (ring) jac_impl<true>(z, J); else jac_impl<false>(z, J);
    }

    // `ChainTangent * W`: GW = _band(W_q); top = (W_q + GW) + W_p, bottom = GW + W_p (chain_tangent.jl:62-78)
    template <bool RING, int KK, class JJ, typename T>
    __device__ __forceinline__ void apply_impl(const JJ& J, T* W) const {
#pragma unroll
        for (int col = 0; col < KK; ++col) {
            T* Wq = W + col * D;
            T v[NS];
#pragma unroll
            for (int j = 0; j < NS; ++j) {
                constexpr int dummy = 0;
                (void)dummy;
                const int kl = L<RING>(j), kr = R<RING>(j);
                T t = static_cast<T>(J.g[j]) * Wq[j];
                if (kl >= 0) t = t + static_cast<T>(J.gl[j]) * Wq[kl];
                if (kr >= 0) t = t + static_cast<T>(J.gr[j]) * Wq[kr];
                v[j] = t;
            }
#pragma unroll
            for (int j = 0; j < NS; ++j) {
                const T wq = Wq[j], wp = Wq[NS + j];
                Wq[j] = (wq + v[j]) + wp;
                Wq[NS + j] = v[j] + wp;
            }
        }
    }
    template <int KK, class JJ, typename T>
    __device__ __forceinline__ void apply(const JJ& J, T* W) const {
        if (ring) apply_impl<true, KK>(J, W); else apply_impl<false, KK>(J, W);
    }

    // forward: p_j' = p_j + (K sin q_j + eps s_j), s_j = (0 + sin(q_j - q_left)) + sin(q_j - q_right); q_j' = q_j + p_j'
    template <bool RING, class JJ>
    __device__ __forceinline__ void forward_impl(double* z, const JJ& J) const {
        double p[NS];
#pragma unroll
        for (int j = 0; j < NS; ++j) {
            double s = 0.0;
            if (L<RING>(j) >= 0) s = s + J.sl[j];
            if (R<RING>(j) >= 0) s = s + J.sr[j];
            p[j] = z[NS + j] + (K * J.sq[j] + eps * s);
        }
#pragma unroll
        for (int j = 0; j < NS; ++j) { z[j] = z[j] + p[j]; z[NS + j] = p[j]; }
    }
    template <class JJ>
    __device__ __forceinline__ void forward(double* z, const JJ& J) const {
        if (ring) forward_impl<true>(z, J); else forward_impl<false>(z, J);
    }
};

// ---- WrappedStandardMapChain (wrapped_standard_map_chain.jl): the chain on the torus with winding counts, state
// (q_1..q_N, p_1..p_N, counts of q, counts of p). The band and the forces are those of the chain at the reduced
// positions (W-E3, :63-67), so `jac` and `apply` are the chain's; only the forward step differs.
template <int NS>
struct SysWrappedChain : SysChain<NS> {
    static constexpr int S = 4 * NS;
    // forward (:117-124, W-E2): p~_j = p_j + F_j(q) reduced with count a_j, n_j' = n_j + a_j; q~_j = q_j + p_j'
    // reduced with count b_j, m_j' = m_j + n_j' + b_j; _guard_counts (:101-107)
    template <bool RING, class JJ>
    __device__ __forceinline__ void forward_w(double* z, const JJ& J) const {
        using B = SysChain<NS>;
        const double tp = 2 * jl_pi();
        double p[NS], nn[NS];
#pragma unroll
        for (int j = 0; j < NS; ++j) {
            double s = 0.0;
            if (B::template L<RING>(j) >= 0) s = s + J.sl[j];
            if (B::template R<RING>(j) >= 0) s = s + J.sr[j];
            double a;
            wrap_reduce(z[NS + j] + (this->K * J.sq[j] + this->eps * s), tp, p[j], a);
            nn[j] = z[3 * NS + j] + a;
        }
        bool ok = true;
#pragma unroll
        for (int j = 0; j < NS; ++j) {
            double q, b;
            wrap_reduce(z[j] + p[j], tp, q, b);
            const double m = z[2 * NS + j] + nn[j] + b;
            z[j] = q; z[NS + j] = p[j]; z[2 * NS + j] = m; z[3 * NS + j] = nn[j];
            ok = ok && fabs(m) < 0x1p53 && fabs(nn[j]) < 0x1p53;
        }
        if (!ok) {
            const double nan = __longlong_as_double(0x7ff8000000000000LL);
#pragma unroll
            for (int i = 0; i < S; ++i) z[i] = nan;
        }
    }
    template <class JJ>
    __device__ __forceinline__ void forward(double* z, const JJ& J) const {
        if (this->ring) forward_w<true>(z, J); else forward_w<false>(z, J);
    }
};

}  // namespace cl
