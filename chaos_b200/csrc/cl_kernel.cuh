// cl_kernel.cuh -- the fused orbit kernel: one orbit per thread, the point in Float64 registers, every tangent
// frame (D x K) and every reducer state in registers, handoffs every tau steps, only final records written to HBM.
//
// It is the device body of the reference's `_orbit_kernel!` (src/Tangent/propagate.jl:32-50) running
// `_orbit_body` (src/Tangent/orbit.jl:44-60): tangent at the old point, frame product, forward; every tau steps the
// status check (`_status`, orbit.jl:3) and the reducer chain (`_apply`, orbit.jl:23-28: every reducer runs, each
// on the W the previous one returned, then `_any_failed`); the final status check only at step N; a launch of
// `steps` steps from global step n0 that carries x, W, states, code and hstep (D44 relaunch), with an orbit that
// failed in an earlier launch frozen.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "../../include/chaoslab_b200.h"
#include "cl_math.cuh"
#include "cl_reducers.cuh"
#include "cl_systems.cuh"

namespace cl {

constexpr int8_t STATUS_OK = 0, STATUS_STATE = 1, STATUS_W = 2, STATUS_REDUCER = 3;

struct KArgs {
    i64 n;                       // orbits in this launch
    i64 n0, steps, N;            // launch window and run length
    int tau;
    int soa;                     // x / W layout: 1 component-major, 0 orbit-major
    const double* x_in;          // n0 == 0: x0; else carried x (may equal x_out)
    double* x_out;
    const double* W_in[CL_MAX_FRAMES];   // n0 == 0: W0 or NULL (seeded); else carried W
    double* W_out[CL_MAX_FRAMES];
    uint64_t* states[CL_MAX_FRAMES];     // orbit-major, Julia layout
    int8_t* code[CL_MAX_FRAMES];
    i64* hstep[CL_MAX_FRAMES];
    uint64_t seed;
    i64 orbit_base;
    RedParams prm[CL_MAX_FRAMES][CL_MAX_REDUCERS];
};

// ---- the reducer chain of one frame as a recursive aggregate --------------------------------------------------------
template <int D, int K, class... Rs> struct Chain;
template <int D, int K> struct Chain<D, K> {
    static constexpr int bytes = 0;
    template <typename T> __device__ __forceinline__ void step(i64, T*, const RedParams*) {}
    __device__ __forceinline__ bool failed() const { return false; }
    __device__ __forceinline__ void load(const uint64_t*) {}
    __device__ __forceinline__ void store(uint64_t*) const {}
    __device__ __forceinline__ void zero() {}
};
template <int D, int K, class R, class... Rs> struct Chain<D, K, R, Rs...> {
    using Head = typename R::template State<D, K>;
    static_assert(sizeof(Head) % 8 == 0, "state size");
    static constexpr int hwords = static_cast<int>(sizeof(Head) / 8);
    static constexpr int bytes = static_cast<int>(sizeof(Head)) + Chain<D, K, Rs...>::bytes;
    Head head;
    Chain<D, K, Rs...> tail;
    template <typename T>
    __device__ __forceinline__ void step(i64 n, T* W, const RedParams* p) {
        R::template step<D, K>(head, n, W, p[0]);
        tail.step(n, W, p + 1);
    }
    __device__ __forceinline__ bool failed() const { return R::template failed<D, K>(head) || tail.failed(); }
    __device__ __forceinline__ void load(const uint64_t* src) {
        uint64_t* h = reinterpret_cast<uint64_t*>(&head);
#pragma unroll
        for (int w = 0; w < hwords; ++w) h[w] = src[w];
        tail.load(src + hwords);
    }
    __device__ __forceinline__ void store(uint64_t* dst) const {
        const uint64_t* h = reinterpret_cast<const uint64_t*>(&head);
#pragma unroll
        for (int w = 0; w < hwords; ++w) dst[w] = h[w];
        tail.store(dst + hwords);
    }
    __device__ __forceinline__ void zero() {
        uint64_t* h = reinterpret_cast<uint64_t*>(&head);
#pragma unroll
        for (int w = 0; w < hwords; ++w) h[w] = 0;
        tail.zero();
    }
};

template <int KK, class... Rs> struct Frame {
    static constexpr int K = KK;
    template <int D> using Chain_ = Chain<D, KK, Rs...>;
};

// ---- seeded Haar frames --------------------------------------------------------------------------------------------
// Key derivation of `initial_deviations` (src/Tangent/initial.jl:27-28): key = _mix(_mix(seed) + orbit); the
// normal variates are this library's own counter stream (Box-Muller on u_t = ((_mix(key + t) >> 11) + 1/2) 2^-53),
// not StableRNGs.jl, then two Gram-Schmidt passes per column. The oracle restates the same stream.
template <int D, int K, typename T>
__device__ __forceinline__ void seeded_frame(uint64_t seed, i64 orbit, T* W) {
    const uint64_t key = mix64(mix64(seed) + static_cast<uint64_t>(orbit));
    double G[D * D];
#pragma unroll
    for (int t = 0; t < D * D; t += 2) {
        const double u1 = (static_cast<double>(mix64(key + static_cast<uint64_t>(t)) >> 11) + 0.5) * 0x1p-53;
        const double u2 = (static_cast<double>(mix64(key + static_cast<uint64_t>(t) + 1) >> 11) + 0.5) * 0x1p-53;
        const double r = sqrt(-2.0 * cl_log(u1));
        double sn, cs; cl_sincos((2 * 3.141592653589793) * u2, &sn, &cs);
        G[t] = r * cs;
        if (t + 1 < D * D) G[t + 1] = r * sn;
    }
#pragma unroll
    for (int j = 0; j < K; ++j) {
#pragma unroll
        for (int pass = 0; pass < 2; ++pass)
#pragma unroll
            for (int i = 0; i < j; ++i) {
                const double c = dotv<D>(G + i * D, G + j * D);
#pragma unroll
                for (int l = 0; l < D; ++l) G[l + j * D] = G[l + j * D] - c * G[l + i * D];
            }
        double s = G[j * D] * G[j * D];
#pragma unroll
        for (int l = 1; l < D; ++l) s = s + G[l + j * D] * G[l + j * D];
        const double nr = sqrt(s);
#pragma unroll
        for (int l = 0; l < D; ++l) G[l + j * D] = G[l + j * D] / nr;
    }
#pragma unroll
    for (int l = 0; l < D * K; ++l) W[l] = static_cast<T>(G[l]);
}

// ---- per-frame register state ---------------------------------------------------------------------------------------
template <int D, typename Real, class F>
struct FrameRegs {
    static constexpr int K = F::K;
    Real W[D * K];
    typename F::template Chain_<D> st;
    int8_t code;
    i64 hstep;
    bool alive;
};

template <int D, int S>
__device__ __forceinline__ bool all_finite_x(const double* x) {
    bool ok = true;
#pragma unroll
    for (int i = 0; i < S; ++i) ok = ok && isfin(x[i]);
    return ok;
}
template <int N, typename Real>
__device__ __forceinline__ bool all_finite(const Real* W) {
    bool ok = true;
#pragma unroll
    for (int i = 0; i < N; ++i) ok = ok && isfin(W[i]);
    return ok;
}

template <int D, int S, typename Real, class F>
__device__ __forceinline__ void frame_load(FrameRegs<D, Real, F>& fr, int f, const KArgs& a, i64 i, bool fresh) {
    constexpr int K = F::K;
    const i64 so = a.soa ? 1 : D * K, sc = a.soa ? a.n : 1;
    if (fresh) {
        if (a.W_in[f]) {
#pragma unroll
            for (int l = 0; l < D * K; ++l) fr.W[l] = static_cast<Real>(a.W_in[f][i * so + l * sc]);
        } else {
            seeded_frame<D, K>(a.seed, a.orbit_base + i + 1, fr.W);
        }
        fr.st.zero();
        fr.code = STATUS_OK;
        fr.hstep = 0;
        fr.alive = true;
    } else {
#pragma unroll
        for (int l = 0; l < D * K; ++l) fr.W[l] = static_cast<Real>(a.W_in[f][i * so + l * sc]);
        constexpr int words = F::template Chain_<D>::bytes / 8;
        if (words > 0) fr.st.load(a.states[f] + i * words);
        fr.code = a.code[f][i];
        fr.hstep = a.hstep[f] ? a.hstep[f][i] : 0;
        fr.alive = fr.code == STATUS_OK;
    }
}

template <int D, int S, typename Real, class F>
__device__ __forceinline__ void frame_store(const FrameRegs<D, Real, F>& fr, int f, const KArgs& a, i64 i) {
    constexpr int K = F::K;
    const i64 so = a.soa ? 1 : D * K, sc = a.soa ? a.n : 1;
#pragma unroll
    for (int l = 0; l < D * K; ++l) a.W_out[f][i * so + l * sc] = static_cast<double>(fr.W[l]);
    constexpr int words = F::template Chain_<D>::bytes / 8;
    if (words > 0) fr.st.store(a.states[f] + i * words);
    a.code[f][i] = fr.code;
    if (a.hstep[f]) a.hstep[f][i] = fr.hstep;
}

// At a handoff: _status, then the chain, then _any_failed (orbit.jl:54-57).
template <int D, int S, typename Real, class F>
__device__ __forceinline__ void frame_handoff(FrameRegs<D, Real, F>& fr, const double* x, i64 n, const RedParams* prm) {
    if (!fr.alive) return;
    constexpr int K = F::K;
    int8_t c = all_finite_x<D, S>(x) ? (all_finite<D * K>(fr.W) ? STATUS_OK : STATUS_W) : STATUS_STATE;
    if (c == STATUS_OK) {
        fr.st.step(n, fr.W, prm);
        if (fr.st.failed()) c = STATUS_REDUCER;
    }
    if (c != STATUS_OK) { fr.code = c; fr.hstep = n; fr.alive = false; }
}

// ---- the kernel ------------------------------------------------------------------------------------------------------
// MINB is the register budget as resident blocks of 128 threads per SM (1: no cap); the tuner picks it per run.
template <class Sys, typename Real, class F0, class F1, class F2, int NF, int MINB>
__global__ void __launch_bounds__(128, MINB) orbit_kernel(const KArgs a, const Sys sys) {
    constexpr int D = Sys::D, S = Sys::S;
    const i64 i = static_cast<i64>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= a.n) return;
    const bool fresh = a.n0 == 0;
    const i64 xso = a.soa ? 1 : S, xsc = a.soa ? a.n : 1;

    double x[S];
    const double* xin = a.x_in;
#pragma unroll
    for (int c = 0; c < S; ++c) x[c] = xin[i * xso + c * xsc];

    FrameRegs<D, Real, F0> fr0;
    FrameRegs<D, Real, F1> fr1;
    FrameRegs<D, Real, F2> fr2;
    frame_load<D, S>(fr0, 0, a, i, fresh);
    if (NF > 1) frame_load<D, S>(fr1, 1, a, i, fresh);
    if (NF > 2) frame_load<D, S>(fr2, 2, a, i, fresh);
    const bool any0 = fr0.alive || (NF > 1 && fr1.alive) || (NF > 2 && fr2.alive);
    if (!any0) return;   // frozen since an earlier launch: nothing is rewritten

    i64 n = a.n0;
    const i64 handoffs = a.steps / a.tau;
    for (i64 h = 0; h < handoffs; ++h) {
        for (int t = 0; t < a.tau; ++t) {
            typename Sys::template JacR<Real> J;
            sys.jac(x, J);
            if (fr0.alive) sys.template apply<F0::K>(J, fr0.W);
            if (NF > 1 && fr1.alive) sys.template apply<F1::K>(J, fr1.W);
            if (NF > 2 && fr2.alive) sys.template apply<F2::K>(J, fr2.W);
            sys.forward(x, J);
        }
        n += a.tau;
        frame_handoff<D, S>(fr0, x, n, a.prm[0]);
        if (NF > 1) frame_handoff<D, S>(fr1, x, n, a.prm[1]);
        if (NF > 2) frame_handoff<D, S>(fr2, x, n, a.prm[2]);
        const bool any = fr0.alive || (NF > 1 && fr1.alive) || (NF > 2 && fr2.alive);
        if (!any) break;
    }
    // orbit.jl:58: the final status check runs only at step N
    if (fr0.alive) { fr0.code = n == a.N ? (all_finite_x<D, S>(x) ? (all_finite<D * F0::K>(fr0.W) ? STATUS_OK : STATUS_W) : STATUS_STATE) : STATUS_OK; fr0.hstep = n; }
    if (NF > 1 && fr1.alive) { fr1.code = n == a.N ? (all_finite_x<D, S>(x) ? (all_finite<D * F1::K>(fr1.W) ? STATUS_OK : STATUS_W) : STATUS_STATE) : STATUS_OK; fr1.hstep = n; }
    if (NF > 2 && fr2.alive) { fr2.code = n == a.N ? (all_finite_x<D, S>(x) ? (all_finite<D * F2::K>(fr2.W) ? STATUS_OK : STATUS_W) : STATUS_STATE) : STATUS_OK; fr2.hstep = n; }

#pragma unroll
    for (int c = 0; c < S; ++c) a.x_out[i * xso + c * xsc] = x[c];
    const bool was0 = fresh || a.code[0][i] == STATUS_OK;
    if (was0) frame_store<D, S>(fr0, 0, a, i);
    if (NF > 1) { const bool was = fresh || a.code[1][i] == STATUS_OK; if (was) frame_store<D, S>(fr1, 1, a, i); }
    if (NF > 2) { const bool was = fresh || a.code[2][i] == STATUS_OK; if (was) frame_store<D, S>(fr2, 2, a, i); }
}

// A placeholder frame for unused slots (never loaded, stepped or stored).
using NoFrame = Frame<1>;

}  // namespace cl
