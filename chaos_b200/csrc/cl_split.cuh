// cl_split.cuh -- IntegratorMap(SplittingMethod(c, d), HenonHeilesFlow(), dt) as a device system: one step of a
// table method (drift c_i dt, then kick d_i dt, first stage first) of the Henon-Heiles flow as a map.
//
// forward is `advance_n(m, flow, z, dt, 1)` (src/Integrators/stepper.jl:27-48): a kick is held back while no drift
// follows, so kicks with no drift between them are applied as one. The tangent is `tangent_advance` with the
// identity frame (stepper.jl:108-118): per stage the drift, then the kick, each one's Jacobian (at the point
// before the sub-step) multiplied onto the frame, and the state advanced without merging kicks. The Jacobians are
// the dense 4 x 4 matrices the reference builds (flow_core.jl:64-72), zeros and ones included, multiplied in the
// StaticArrays order with every fusion explicit (the chain of fused_product), so the results are the oracle's
// bit for bit. The table is at most CL_MAX_STAGES stages; its weights are read from the kernel's parameters.
#pragma once

#include "cl_registry.cuh"

namespace cl {

struct SplitJac { double T[16]; };
struct SplitJacF { float T[16]; double xn[4]; };   // mixed kernels: the step's tangent in Float32 and the new point

struct SysSplitHH {
    static constexpr int D = 4, S = 4;
    using Jac = SplitJac;
    template <typename R> using JacR = typename std::conditional<sizeof(R) == 8, SplitJac, SplitJacF>::type;
    double dt;
    int n;
    int corr;       // CorrectedMethod: the corrector kick before and after every step
    double kap;     // its kappa = dt^3 eps^2 c / 2 (stepper.jl:131-134), eps = perturbation_scale = 1 here
    double c[CL_MAX_STAGES], d[CL_MAX_STAGES];

    // force (flow_models.jl:102): (q1 + 2 q1 q2, q2 + q1^2 - q2^2), left to right as Julia evaluates it
    static __device__ __forceinline__ void force(double q1, double q2, double& F1, double& F2) {
        F1 = q1 + (2 * q1) * q2;
        F2 = (q2 + q1 * q1) - q2 * q2;
    }
    // drift (flow_core.jl:59): q += t p; kick (flow_core.jl:60): p -= t grad V(q)
    static __device__ __forceinline__ void drift(double* z, double t) { z[0] = z[0] + t * z[2]; z[1] = z[1] + t * z[3]; }
    static __device__ __forceinline__ void kick(double* z, double t) {
        double F1, F2;
        force(z[0], z[1], F1, F2);
        z[2] = z[2] - t * F1;
        z[3] = z[3] - t * F2;
    }
    // corrector_force (flow_models.jl:106): 2 (Hs g), Hs the force Jacobian, g the force, the SMatrix-vector
    // product fused as StaticArrays unrolls it
    static __device__ __forceinline__ void corrector_force(double q1, double q2, double& C1, double& C2) {
        double F1, F2;
        force(q1, q2, F1, F2);
        const double h11 = 1 + 2 * q2, h21 = 2 * q1, h12 = 2 * q1, h22 = 1 - 2 * q2;
        C1 = 2 * fma(h12, F2, h11 * F1);
        C2 = 2 * fma(h22, F2, h21 * F1);
    }
    // _corrector_kick (stepper.jl:136): p + kappa * corrector_force
    __device__ __forceinline__ void corrector_kick(double* z) const {
        double C1, C2;
        corrector_force(z[0], z[1], C1, C2);
        z[2] = z[2] + kap * C1;
        z[3] = z[3] + kap * C2;
    }
    // _corrector_jacobian (stepper.jl:137-140): [[I, 0], [kappa Hc, I]], Hc = corrector_hessian
    // (flow_models.jl:107-112) = 2 (Hs Hs + g1 T1 + g2 T2), T1 = [0 2; 2 0], T2 = [2 0; 0 -2]
    __device__ __forceinline__ void corrector_jacobian(const double* z, double* J) const {
        double F1, F2;
        force(z[0], z[1], F1, F2);
        const double h[4] = {1 + 2 * z[1], 2 * z[0], 2 * z[0], 1 - 2 * z[1]};   // column-major Hs
        const double t1[4] = {0, 2, 2, 0}, t2[4] = {2, 0, 0, -2};
        double hc[4];
#pragma unroll
        for (int j = 0; j < 2; ++j)
#pragma unroll
            for (int i = 0; i < 2; ++i) {
                const double hh = fma(h[i + 2], h[1 + 2 * j], h[i] * h[2 * j]);
                hc[i + 2 * j] = 2 * ((hh + F1 * t1[i + 2 * j]) + F2 * t2[i + 2 * j]);
            }
        const double Jv[16] = {1, 0, kap * hc[0], kap * hc[1], 0, 1, kap * hc[2], kap * hc[3], 0, 0, 1, 0, 0, 0, 0, 1};
#pragma unroll
        for (int l = 0; l < 16; ++l) J[l] = Jv[l];
    }
    // W <- J W for a 4 x 4 frame, both column-major, entry (i, j): J[i,0] W[0,j], then fma over q = 1..3
    static __device__ __forceinline__ void mul4(const double* J, double* W) {
        double Wn[16];
#pragma unroll
        for (int j = 0; j < 4; ++j)
#pragma unroll
            for (int i = 0; i < 4; ++i) {
                double acc = J[i] * W[4 * j];
#pragma unroll
                for (int q = 1; q < 4; ++q) acc = fma(J[i + 4 * q], W[q + 4 * j], acc);
                Wn[i + 4 * j] = acc;
            }
#pragma unroll
        for (int l = 0; l < 16; ++l) W[l] = Wn[l];
    }

    __device__ __forceinline__ void jac(const double* x, SplitJac& Jc) const {
        double z[4] = {x[0], x[1], x[2], x[3]};
        double* W = Jc.T;
#pragma unroll
        for (int l = 0; l < 16; ++l) W[l] = (l % 5 == 0) ? 1.0 : 0.0;
        if (corr) {   // tangent_advance(::CorrectedMethod) (stepper.jl:154-160): the corrector's Jacobian, its kick
            double J[16];
            corrector_jacobian(z, J);
            mul4(J, W);
            corrector_kick(z);
        }
#pragma unroll 1
        for (int i = 0; i < n; ++i) {
            const double ci = c[i], di = d[i];
            if (ci != 0.0) {
                // drift_jacobian (flow_core.jl:64-67): [[I, t I], [0, I]] with its entries t * 1 and t * 0
                const double t = ci * dt;
                const double J[16] = {1, 0, 0, 0, 0, 1, 0, 0, t * 1.0, t * 0.0, 1, 0, t * 0.0, t * 1.0, 0, 1};
                mul4(J, W);
                drift(z, t);
            }
            if (di != 0.0) {
                // kick_jacobian (flow_core.jl:68-72) at the pre-kick point: [[I, 0], [(-t) Hs, I]], Hs the
                // force Jacobian (flow_models.jl:103)
                const double t = di * dt, mt = -t;
                const double h11 = 1 + 2 * z[1], h21 = 2 * z[0], h12 = 2 * z[0], h22 = 1 - 2 * z[1];
                const double J[16] = {1, 0, mt * h11, mt * h21, 0, 1, mt * h12, mt * h22, 0, 0, 1, 0, 0, 0, 0, 1};
                mul4(J, W);
                kick(z, t);
            }
        }
        if (corr) {
            double J[16];
            corrector_jacobian(z, J);
            mul4(J, W);
        }
    }
    template <int KK, typename T>
    __device__ __forceinline__ void apply(const SplitJac& Jc, T* W) const { fused_dense<4, KK>(Jc.T, W); }

    // the p rows of the Float32 product += [a c; b dd] times its q rows
    static __device__ __forceinline__ void lower(float* T, float a, float b, float c, float dd) {
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const float q1 = T[4 * j], q2 = T[4 * j + 1];
            T[4 * j + 2] = __fmaf_rn(a, q1, __fmaf_rn(c, q2, T[4 * j + 2]));
            T[4 * j + 3] = __fmaf_rn(b, q1, __fmaf_rn(dd, q2, T[4 * j + 3]));
        }
    }
    // Mixed kernels: one pass along the forward step (advance_n's merged kicks, Float64 points) that also builds
    // the step's tangent in Float32 from the blocks of the Jacobians of the sub-steps it takes -- a drift adds
    // t * (p rows) to the q rows, a kick subtracts t * Hs (q rows) from the p rows (a merged kick's Jacobian is the
    // product of its parts' at the same q), the corrector adds kappa * Hc (q rows) -- instead of the plain kernel's
    // separate unmerged tangent pass with dense 4 x 4 Float64 products.
    __device__ __forceinline__ void jac(const double* x, SplitJacF& Jc) const {
        double z[4] = {x[0], x[1], x[2], x[3]};
        float* T = Jc.T;
#pragma unroll
        for (int l = 0; l < 16; ++l) T[l] = (l % 5 == 0) ? 1.0f : 0.0f;
        if (corr) {
            double J[16];
            corrector_jacobian(z, J);
            lower(T, static_cast<float>(J[2]), static_cast<float>(J[3]), static_cast<float>(J[6]), static_cast<float>(J[7]));
            corrector_kick(z);
        }
        double pend = 0.0;
#pragma unroll 1
        for (int i = 0; i < n; ++i) {
            const double ci = c[i];
            if (ci != 0.0) {
                if (pend != 0.0) { kick_t(z, T, pend * dt); pend = 0.0; }
                const float t = static_cast<float>(ci * dt);
#pragma unroll
                for (int j = 0; j < 4; ++j) {
                    T[4 * j] = __fmaf_rn(t, T[4 * j + 2], T[4 * j]);
                    T[4 * j + 1] = __fmaf_rn(t, T[4 * j + 3], T[4 * j + 1]);
                }
                drift(z, ci * dt);
            }
            pend = pend + d[i];
        }
        if (pend != 0.0) kick_t(z, T, pend * dt);
        if (corr) {
            double J[16];
            corrector_jacobian(z, J);
            lower(T, static_cast<float>(J[2]), static_cast<float>(J[3]), static_cast<float>(J[6]), static_cast<float>(J[7]));
            corrector_kick(z);
        }
#pragma unroll
        for (int l = 0; l < 4; ++l) Jc.xn[l] = z[l];
    }
    // a kick of time t on the Float64 point and its Jacobian [[I, 0], [-t Hs, I]] on the Float32 tangent
    static __device__ __forceinline__ void kick_t(double* z, float* T, double t) {
        const float mt = static_cast<float>(-t);
        const float h11 = static_cast<float>(1 + 2 * z[1]), h12 = static_cast<float>(2 * z[0]);
        const float h22 = static_cast<float>(1 - 2 * z[1]);
        lower(T, mt * h11, mt * h12, mt * h12, mt * h22);
        kick(z, t);
    }
    template <int KK>
    __device__ __forceinline__ void apply(const SplitJacF& Jc, float* W) const { fused_dense<4, KK>(Jc.T, W); }
    __device__ __forceinline__ void forward(double* x, const SplitJac&) const { step(x); }
    __device__ __forceinline__ void forward(double* x, const SplitJacF& J) const {   // the point jac took the step to
#pragma unroll
        for (int l = 0; l < 4; ++l) x[l] = J.xn[l];
    }
    // one step of advance_n; a corrected method (stepper.jl:142-152): kick, the base step with its own merged
    // kicks, kick (no merging across the corrector)
    __device__ __forceinline__ void step(double* x) const {
        if (corr) corrector_kick(x);
        double pend = 0.0;
#pragma unroll 1
        for (int i = 0; i < n; ++i) {
            const double ci = c[i];
            if (ci != 0.0) {
                if (pend != 0.0) { kick(x, pend * dt); pend = 0.0; }
                drift(x, ci * dt);
            }
            pend = pend + d[i];
        }
        if (pend != 0.0) kick(x, pend * dt);
        if (corr) corrector_kick(x);
    }
};

template <> struct SysMaker<SysSplitHH> {
    static SysSplitHH make(const cl_run& r, const double*) {
        SysSplitHH s;
        s.dt = r.sys.dt;
        s.n = r.sys.n_stages;
        s.corr = r.sys.corrector;
        // kappa = tau * tau * tau * (eps * eps) * c / 2 left to right, eps * eps the integer 1
        s.kap = r.sys.corrector ? (((r.sys.dt * r.sys.dt) * r.sys.dt) * r.sys.eps) / 2 : 0.0;
        for (int i = 0; i < CL_MAX_STAGES; ++i) {
            s.c[i] = i < s.n ? r.sys.stage_c[i] : 0.0;
            s.d[i] = i < s.n ? r.sys.stage_d[i] : 0.0;
        }
        return s;
    }
};

}  // namespace cl
