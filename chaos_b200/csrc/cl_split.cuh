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

struct SysSplitHH {
    static constexpr int D = 4, S = 4;
    using Jac = SplitJac;
    template <typename R> using JacR = SplitJac;
    double dt;
    int n;
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
    }
    template <int KK, typename T>
    __device__ __forceinline__ void apply(const SplitJac& Jc, T* W) const { fused_dense<4, KK>(Jc.T, W); }
    __device__ __forceinline__ void forward(double* x, const SplitJac&) const {
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
    }
};

template <> struct SysMaker<SysSplitHH> {
    static SysSplitHH make(const cl_run& r, const double*) {
        SysSplitHH s;
        s.dt = r.sys.dt;
        s.n = r.sys.n_stages;
        for (int i = 0; i < CL_MAX_STAGES; ++i) {
            s.c[i] = i < s.n ? r.sys.stage_c[i] : 0.0;
            s.d[i] = i < s.n ? r.sys.stage_d[i] : 0.0;
        }
        return s;
    }
};

}  // namespace cl
