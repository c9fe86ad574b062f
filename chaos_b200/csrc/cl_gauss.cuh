// cl_gauss.cuh -- IntegratorMap(Gauss(Float64, 3; tol), HenonHeilesFlow(), dt) as a device system: one step of the
// 3-stage Gauss-Legendre collocation method (order 6) on the Henon-Heiles flow, and the exact Jacobian of that step.
//
// Follows src/Integrators/gauss.jl operation for operation:
//   _gauss_core (:122-141): initial stages Y_i = z + (h sum_j Ahi_ij) f(z); fixed-point iteration F = f(Y),
//     Y_i = z + (0 + h dotcomp(Ahi_i, Alo_i, F)) until the increment is 0 or stops decreasing (k >= 2), at most
//     maxiter; accepted when the increment is within the bound (tol, or 8 eps max(1, |Y|)); update h dotcomp(b, F)
//     with F from the last iteration. dotcomp (:91-101) is the compensated dot product (TwoProd by fma, TwoSum).
//   tangent_advance (:176-192) with W = I (IntegratorMap.tangent, integrator_map.jl:21): M = I - h (A (x) J), A =
//     Ahi + Alo, M \ repeat(I, 3, 1), T = I + sum_i (h (bhi_i + blo_i)) (J_i dY_i). The solve is the unblocked LU
//     with partial pivoting and the triangular solves in the dgetf2 / dgetrs order, J_i dY_i in the dgemm order
//     (Julia runs OpenBLAS there); the CPU oracle restates the same order.
//   `forward` reruns the same core on the same point (advance_n, :149-158): it gives the same bits, so the step
//     computes it once.
// The mixed kernels run the same Float64 step (fixed point, stages, update) and solve the tangent's linear system
// in Float32 (tangent32, below); the frames are Float32.
#pragma once

#include "cl_math.cuh"
#include "cl_registry.cuh"
#include "cl_systems.cuh"

namespace cl {

// vector_field (flow_core.jl:78) with the Henon-Heiles force (flow_models.jl:102)
__device__ __forceinline__ void hh_vf(const double* z, double* f) {
    const double F1 = z[0] + 2 * z[0] * z[1];
    const double F2 = (z[1] + z[0] * z[0]) - z[1] * z[1];
    f[0] = z[2]; f[1] = z[3]; f[2] = -F1; f[3] = -F2;
}

struct GaussJac { double T[16]; double xn[4]; };
struct GaussJacF { float T[16]; double xn[4]; };   // mixed kernels: the step's tangent in Float32

struct SysGauss3HH {
    static constexpr int D = 4, S = 4;
    using Jac = GaussJac;
    template <typename R> using JacR = typename std::conditional<sizeof(R) == 8, GaussJac, GaussJacF>::type;
    double h, tol;
    int maxiter;

    static __device__ __forceinline__ double Ahi(int i, int j) {
        const double a[9] = {CL_GAUSS3_AHI_00, CL_GAUSS3_AHI_01, CL_GAUSS3_AHI_02, CL_GAUSS3_AHI_10, CL_GAUSS3_AHI_11,
                             CL_GAUSS3_AHI_12, CL_GAUSS3_AHI_20, CL_GAUSS3_AHI_21, CL_GAUSS3_AHI_22};
        return a[i * 3 + j];
    }
    static __device__ __forceinline__ double Alo(int i, int j) {
        const double a[9] = {CL_GAUSS3_ALO_00, CL_GAUSS3_ALO_01, CL_GAUSS3_ALO_02, CL_GAUSS3_ALO_10, CL_GAUSS3_ALO_11,
                             CL_GAUSS3_ALO_12, CL_GAUSS3_ALO_20, CL_GAUSS3_ALO_21, CL_GAUSS3_ALO_22};
        return a[i * 3 + j];
    }
    static __device__ __forceinline__ double bhi(int i) {
        const double b[3] = {CL_GAUSS3_BHI_0, CL_GAUSS3_BHI_1, CL_GAUSS3_BHI_2};
        return b[i];
    }
    static __device__ __forceinline__ double blo(int i) {
        const double b[3] = {CL_GAUSS3_BLO_0, CL_GAUSS3_BLO_1, CL_GAUSS3_BLO_2};
        return b[i];
    }

    // _dot_comp per component (gauss.jl:91-101): w runs hi_1, lo_1, hi_2, lo_2, hi_3, lo_3.
    template <bool STAGE>
    static __device__ __forceinline__ void dot_comp(int i, const double F[3][4], double* out) {
#pragma unroll
        for (int l = 0; l < 4; ++l) {
            double s = 0.0, c = 0.0;
#pragma unroll
            for (int j = 0; j < 3; ++j)
#pragma unroll
                for (int hh = 0; hh < 2; ++hh) {
                    const double w = STAGE ? (hh == 0 ? Ahi(i, j) : Alo(i, j)) : (hh == 0 ? bhi(j) : blo(j));
                    const double p = w * F[j][l];
                    const double pe = fma(w, F[j][l], -p);
                    const double t = s + p;
                    const double bb = t - s;
                    const double se = (s - (t - bb)) + (p - bb);
                    s = t;
                    c = c + (se + pe);
                }
            out[l] = s + c;
        }
    }

    // _gauss_core (compensated, e = 0); returns ok, writes the increment and the final stages.
    __device__ __forceinline__ bool core(const double* z, double* inc, double Y[3][4]) const {
        double f0[4];
        hh_vf(z, f0);
#pragma unroll
        for (int i = 0; i < 3; ++i) {
            const double ci = h * ((Ahi(i, 0) + Ahi(i, 1)) + Ahi(i, 2));
#pragma unroll
            for (int l = 0; l < 4; ++l) Y[i][l] = z[l] + ci * f0[l];
        }
        double F[3][4];
#pragma unroll
        for (int i = 0; i < 3; ++i)
#pragma unroll
            for (int l = 0; l < 4; ++l) F[i][l] = f0[l];
        double delta = 0.0, prev = __longlong_as_double(0x7ff0000000000000LL);
        bool stopped = false;
        int k = 0;
        while (k < maxiter && !stopped) {
            k += 1;
#pragma unroll
            for (int i = 0; i < 3; ++i) hh_vf(Y[i], F[i]);
            double dm = 0.0;
#pragma unroll
            for (int i = 0; i < 3; ++i) {
                double ss[4];
                dot_comp<true>(i, F, ss);
                double m = 0.0;
#pragma unroll
                for (int l = 0; l < 4; ++l) {
                    const double yn = z[l] + (0.0 + h * ss[l]);
                    const double a = fabs(yn - Y[i][l]);
                    m = l == 0 ? a : jl_max(m, a);
                    Y[i][l] = yn;
                }
                dm = i == 0 ? m : jl_max(dm, m);
            }
            delta = dm;
            if (!isfin(delta)) break;
            stopped = (delta == 0.0) || (k >= 2 && delta >= prev);
            prev = delta;
        }
        double bound;
        if (isnan(tol)) {
            double mn = 0.0;
#pragma unroll
            for (int i = 0; i < 3; ++i) {
                double m = fabs(Y[i][0]);
#pragma unroll
                for (int l = 1; l < 4; ++l) m = jl_max(m, fabs(Y[i][l]));
                mn = i == 0 ? m : jl_max(mn, m);
            }
            bound = 8 * 0x1p-52 * jl_max(1.0, mn);
        } else {
            bound = tol;
        }
        const bool ok = stopped && isfin(delta) && delta <= bound;
        double us[4];
        dot_comp<false>(0, F, us);
#pragma unroll
        for (int l = 0; l < 4; ++l) inc[l] = h * us[l];
        return ok;
    }

    // vector_field_jacobian (flow_core.jl:79-83) at a stage: [[0, I], [-Hs, 0]] with the Henon-Heiles Hessian
    // Hs = [[1 + 2 q2, 2 q1], [2 q1, 1 - 2 q2]] (flow_models.jl:103); column-major 4 x 4.
    static __device__ __forceinline__ void hh_jac(const double* y, double* Jm) {
        const double h11 = 1 + 2 * y[1], h21 = 2 * y[0], h12 = 2 * y[0], h22 = 1 - 2 * y[1];
        Jm[0] = 0; Jm[1] = 0; Jm[2] = -h11; Jm[3] = -h21;
        Jm[4] = 0; Jm[5] = 0; Jm[6] = -h12; Jm[7] = -h22;
        Jm[8] = 1; Jm[9] = 0; Jm[10] = 0; Jm[11] = 0;
        Jm[12] = 0; Jm[13] = 1; Jm[14] = 0; Jm[15] = 0;
    }

    // The 12 x 12 solve of tangent_advance and the assembly of T (Float64, reference order).
    static __device__ __noinline__ void tangent64(const double* Yflat, double hstep, double* T) {
        double Jm[3][16];
        for (int i = 0; i < 3; ++i) hh_jac(Yflat + 4 * i, Jm[i]);
        double M[144], B[48];
        for (int c = 0; c < 12; ++c)
            for (int r = 0; r < 12; ++r) M[r + 12 * c] = r == c ? 1.0 : 0.0;
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j) {
                const double f = hstep * (Ahi(i, j) + Alo(i, j));
                for (int c = 0; c < 4; ++c)
                    for (int r = 0; r < 4; ++r) {
                        const int at = (i * 4 + r) + 12 * (j * 4 + c);
                        M[at] = M[at] - f * Jm[j][r + 4 * c];
                    }
            }
        for (int c = 0; c < 4; ++c)
            for (int r = 0; r < 12; ++r) B[r + 12 * c] = (r % 4) == c ? 1.0 : 0.0;
        int ipiv[12];
        for (int j = 0; j < 12; ++j) {
            int p = j;
            double pm = fabs(M[j + 12 * j]);
            for (int i = j + 1; i < 12; ++i) {
                const double av = fabs(M[i + 12 * j]);
                if (av > pm) { pm = av; p = i; }
            }
            ipiv[j] = p;
            if (M[p + 12 * j] != 0.0) {
                if (p != j)
                    for (int c = 0; c < 12; ++c) {
                        const double t = M[j + 12 * c];
                        M[j + 12 * c] = M[p + 12 * c];
                        M[p + 12 * c] = t;
                    }
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
            if (ipiv[j] != j)
                for (int c = 0; c < 4; ++c) {
                    const double t = B[j + 12 * c];
                    B[j + 12 * c] = B[ipiv[j] + 12 * c];
                    B[ipiv[j] + 12 * c] = t;
                }
        for (int c = 0; c < 4; ++c) {
            double* bc = B + 12 * c;
            for (int k = 0; k < 12; ++k)
                if (bc[k] != 0.0)
                    for (int i = k + 1; i < 12; ++i) bc[i] = bc[i] - bc[k] * M[i + 12 * k];
            for (int k = 11; k >= 0; --k)
                if (bc[k] != 0.0) {
                    bc[k] = bc[k] / M[k + 12 * k];
                    for (int i = 0; i < k; ++i) bc[i] = bc[i] - bc[k] * M[i + 12 * k];
                }
        }
        double Wn[16];
        for (int l = 0; l < 16; ++l) Wn[l] = (l % 4) == (l / 4) ? 1.0 : 0.0;
        for (int i = 0; i < 3; ++i) {
            double P[16];
            for (int jj = 0; jj < 4; ++jj) {
                for (int ii = 0; ii < 4; ++ii) P[ii + 4 * jj] = 0.0;
                for (int l = 0; l < 4; ++l) {
                    const double temp = B[(i * 4 + l) + 12 * jj];
                    for (int ii = 0; ii < 4; ++ii) P[ii + 4 * jj] = P[ii + 4 * jj] + temp * Jm[i][ii + 4 * l];
                }
            }
            const double f = hstep * (bhi(i) + blo(i));
            for (int l = 0; l < 16; ++l) Wn[l] = Wn[l] + f * P[l];
        }
        for (int l = 0; l < 16; ++l) T[l] = Wn[l];
    }

    __device__ __forceinline__ void jac(const double* x, GaussJac& Jc) const {
        double inc[4], Y[3][4];
        const bool ok = core(x, inc, Y);
        if (!ok) {
            const double nan = __longlong_as_double(0x7ff8000000000000LL);
#pragma unroll
            for (int l = 0; l < 16; ++l) Jc.T[l] = nan;
#pragma unroll
            for (int l = 0; l < 4; ++l) Jc.xn[l] = nan;
            return;
        }
        tangent64(&Y[0][0], h, Jc.T);
#pragma unroll
        for (int l = 0; l < 4; ++l) Jc.xn[l] = x[l] + inc[l];
    }
    template <int KK, typename T>
    __device__ __forceinline__ void apply(const GaussJac& Jc, T* W) const { fused_dense<4, KK>(Jc.T, W); }

    // Mixed kernels: the Float64 step (fixed point, stages, update) as above, and the tangent's linear system
    // (I - h A (x) J) dY = 1 (x) I in Float32 by its fixed-point form dY = 1 (x) I + h (A (x) J) dY, which converges
    // geometrically for h ||A|| ||J|| < 1 (0.01 x 0.5 x ~2 at the Henon-Heiles workload: ~2 digits a sweep), with
    // the stage Jacobians J_i = [[0, I], [-Hs_i, 0]] applied by blocks; T = I + sum_i h b_i J_i dY_i. Everything is
    // indexed statically (registers, no local-memory LU). A system that has not converged in 24 sweeps takes the
    // Float64 LU of the plain kernel.
    static __device__ __forceinline__ void tangent32(const double Y[3][4], double hstep, float* T) {
        float hs[3][3];
        float a[3][3], bw[3];
#pragma unroll
        for (int i = 0; i < 3; ++i) {
            hs[i][0] = static_cast<float>(1 + 2 * Y[i][1]);
            hs[i][1] = static_cast<float>(2 * Y[i][0]);
            hs[i][2] = static_cast<float>(1 - 2 * Y[i][1]);
            bw[i] = static_cast<float>(hstep * (bhi(i) + blo(i)));
#pragma unroll
            for (int j = 0; j < 3; ++j) a[i][j] = static_cast<float>(hstep * (Ahi(i, j) + Alo(i, j)));
        }
        float dY[3][16];
#pragma unroll
        for (int i = 0; i < 3; ++i)
#pragma unroll
            for (int l = 0; l < 16; ++l) dY[i][l] = (l % 5 == 0) ? 1.0f : 0.0f;
        bool conv = false;
#pragma unroll 1
        for (int it = 0; it < 24 && !conv; ++it) {
            float JdY[3][16];
#pragma unroll
            for (int j = 0; j < 3; ++j)
#pragma unroll
                for (int c = 0; c < 4; ++c) {
                    const float q1 = dY[j][4 * c], q2 = dY[j][4 * c + 1];
                    JdY[j][4 * c] = dY[j][4 * c + 2];
                    JdY[j][4 * c + 1] = dY[j][4 * c + 3];
                    JdY[j][4 * c + 2] = -__fmaf_rn(hs[j][0], q1, hs[j][1] * q2);
                    JdY[j][4 * c + 3] = -__fmaf_rn(hs[j][1], q1, hs[j][2] * q2);
                }
            float change = 0.0f, scale = 0.0f;
#pragma unroll
            for (int i = 0; i < 3; ++i)
#pragma unroll
                for (int l = 0; l < 16; ++l) {
                    float v = (l % 5 == 0) ? 1.0f : 0.0f;
                    v = __fmaf_rn(a[i][0], JdY[0][l], v);
                    v = __fmaf_rn(a[i][1], JdY[1][l], v);
                    v = __fmaf_rn(a[i][2], JdY[2][l], v);
                    change = fmaxf(change, fabsf(v - dY[i][l]));
                    scale = fmaxf(scale, fabsf(v));
                    dY[i][l] = v;
                }
            conv = change <= 0x1p-24f * scale;
        }
        if (!conv) {
            double T64[16];
            tangent64(&Y[0][0], hstep, T64);
#pragma unroll
            for (int l = 0; l < 16; ++l) T[l] = static_cast<float>(T64[l]);
            return;
        }
#pragma unroll
        for (int l = 0; l < 16; ++l) T[l] = (l % 5 == 0) ? 1.0f : 0.0f;
#pragma unroll
        for (int i = 0; i < 3; ++i)
#pragma unroll
            for (int c = 0; c < 4; ++c) {
                const float q1 = dY[i][4 * c], q2 = dY[i][4 * c + 1];
                T[4 * c] = __fmaf_rn(bw[i], dY[i][4 * c + 2], T[4 * c]);
                T[4 * c + 1] = __fmaf_rn(bw[i], dY[i][4 * c + 3], T[4 * c + 1]);
                T[4 * c + 2] = __fmaf_rn(bw[i], -__fmaf_rn(hs[i][0], q1, hs[i][1] * q2), T[4 * c + 2]);
                T[4 * c + 3] = __fmaf_rn(bw[i], -__fmaf_rn(hs[i][1], q1, hs[i][2] * q2), T[4 * c + 3]);
            }
    }
    __device__ __forceinline__ void jac(const double* x, GaussJacF& Jc) const {
        double inc[4], Y[3][4];
        const bool ok = core(x, inc, Y);
        if (!ok) {
            const double nan = __longlong_as_double(0x7ff8000000000000LL);
#pragma unroll
            for (int l = 0; l < 16; ++l) Jc.T[l] = __int_as_float(0x7fc00000);
#pragma unroll
            for (int l = 0; l < 4; ++l) Jc.xn[l] = nan;
            return;
        }
        tangent32(Y, h, Jc.T);
#pragma unroll
        for (int l = 0; l < 4; ++l) Jc.xn[l] = x[l] + inc[l];
    }
    template <int KK>
    __device__ __forceinline__ void apply(const GaussJacF& Jc, float* W) const { fused_dense<4, KK>(Jc.T, W); }

    template <class JJ>
    __device__ __forceinline__ void forward(double* x, const JJ& Jc) const {
#pragma unroll
        for (int l = 0; l < 4; ++l) x[l] = Jc.xn[l];
    }
};

template <> struct SysMaker<SysGauss3HH> {
    static SysGauss3HH make(const cl_run& r, const double*) {
        SysGauss3HH s;
        s.h = r.sys.dt;
        s.tol = r.sys.gauss_tol;
        s.maxiter = r.sys.gauss_maxiter;
        return s;
    }
};

}  // namespace cl
