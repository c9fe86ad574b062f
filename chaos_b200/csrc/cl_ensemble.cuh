// cl_ensemble.cuh -- the batched uneven ensemble: one persistent kernel per dimension class that takes orbits from
// a device work queue, each orbit with its own map parameter K, its own length N_i and an escape stop.
//
// The reference's `propagate` has one N and one system per call and stops an orbit only on a non-finite value; the
// ensemble generalises it per orbit. Orbit i is, bit for bit, the reference call `propagate_orbit(sys(K_i), x0_i,
// W0_i, N_i', tau, reducers)` (src/Tangent/orbit.jl:85-99) where N_i' is N_i, or the first handoff at which
// max_j |p_j| > escape (the orbit then reports STATUS_ESCAPED = 4 instead of 0; x, W and the reducer states are
// those of the N_i' run). Orbits are handed out in the caller's order (longest first balances the load): one
// atomicAdd per warp claims 32 consecutive queue slots, so a warp's lanes run orbits of similar length. No thread
// ever waits on another: the queue is a counter, not a barrier.
#pragma once

#include "cl_kernel.cuh"
#include "cl_registry.cuh"

namespace cl {

constexpr int8_t STATUS_ESCAPED = 4;

struct EArgs {
    i64 n;                        // orbits of this class
    unsigned long long* counter;  // queue head (zeroed before the launch)
    const i64* order;             // queue: orbit indices, longest first
    const double* x_in;           // AoS n x S
    double* x_out;
    const double* W_in;           // AoS n x D*K, NULL = seeded frames
    double* W_out;
    uint64_t* states;
    int8_t* code;
    i64* hstep;
    const double* Kp;             // per-orbit K (NULL = the system's)
    const i64* Np;                // per-orbit N (NULL = N)
    i64 N;
    int tau;
    double escape;                // <= 0: off
    uint64_t seed;
    i64 orbit_base;
    RedParams prm[CL_MAX_REDUCERS];
};

template <class Sys> struct HasK { static constexpr bool value = false; };
template <> struct HasK<SysStandard> { static constexpr bool value = true; };
template <> struct HasK<SysWrapped> { static constexpr bool value = true; };
template <int NS> struct HasK<SysChain<NS>> { static constexpr bool value = true; };

// max_j |p_j| over the momenta of the state (the second half of (q, p); (x, p) for the standard map)
template <class Sys>
__device__ __forceinline__ double max_abs_p(const double* x) {
    constexpr int D = Sys::D;
    double m = fabs(x[D / 2]);
#pragma unroll
    for (int j = D / 2 + 1; j < D; ++j) m = fmax(m, fabs(x[j]));
    return m;
}

template <class Sys, typename Real, class F, int TAU_UNROLL, int MINB>
__global__ void __launch_bounds__(128, MINB) ensemble_kernel(const EArgs a, Sys sys0) {
    constexpr int D = Sys::D, S = Sys::S, K = F::K;
    const int lane = threadIdx.x & 31;
    for (;;) {
        unsigned long long base = 0;
        if (lane == 0) base = atomicAdd(a.counter, 32ULL);
        base = __shfl_sync(0xffffffffu, base, 0);
        if (base >= static_cast<unsigned long long>(a.n)) return;
        const i64 slot = static_cast<i64>(base) + lane;
        if (slot >= a.n) continue;
        const i64 i = a.order ? a.order[slot] : slot;

        Sys sys = sys0;
        if constexpr (HasK<Sys>::value) { if (a.Kp) sys.K = a.Kp[i]; }
        const i64 Ni = a.Np ? a.Np[i] : a.N;
        double x[S];
#pragma unroll
        for (int c = 0; c < S; ++c) x[c] = a.x_in[i * S + c];
        FrameRegs<D, Real, F> fr;
        if (a.W_in) {
#pragma unroll
            for (int l = 0; l < D * K; ++l) fr.W[l] = static_cast<Real>(a.W_in[i * D * K + l]);
        } else {
            seeded_frame<D, K>(a.seed, a.orbit_base + i + 1, fr.W);
        }
        fr.st.zero();
        fr.code = STATUS_OK;
        fr.hstep = 0;
        fr.alive = true;
        i64 n = 0;
        bool escaped = false;
        const i64 handoffs = Ni / a.tau;
        for (i64 h = 0; h < handoffs; ++h) {
            if (TAU_UNROLL > 1) {
#pragma unroll
                for (int t = 0; t < TAU_UNROLL; ++t) {
                    typename Sys::template JacR<Real> J;
                    sys.jac(x, J);
                    sys.template apply<K>(J, fr.W);
                    sys.forward(x, J);
                }
            } else {
                for (int t = 0; t < a.tau; ++t) {
                    typename Sys::template JacR<Real> J;
                    sys.jac(x, J);
                    sys.template apply<K>(J, fr.W);
                    sys.forward(x, J);
                }
            }
            n += a.tau;
            frame_handoff<D, S>(fr, x, n, a.prm);
            if (!fr.alive) break;
            if (a.escape > 0.0 && max_abs_p<Sys>(x) > a.escape) { escaped = true; break; }
        }
        if (fr.alive) {
            const bool fin = all_finite_x<D, S>(x) && all_finite<D * K>(fr.W);
            fr.code = escaped ? (fin ? STATUS_ESCAPED : (all_finite_x<D, S>(x) ? STATUS_W : STATUS_STATE))
                              : (n == Ni ? (fin ? STATUS_OK : (all_finite_x<D, S>(x) ? STATUS_W : STATUS_STATE)) : STATUS_OK);
            fr.hstep = n;
        }
#pragma unroll
        for (int c = 0; c < S; ++c) a.x_out[i * S + c] = x[c];
#pragma unroll
        for (int l = 0; l < D * K; ++l) a.W_out[i * D * K + l] = static_cast<double>(fr.W[l]);
        constexpr int words = F::template Chain_<D>::bytes / 8;
        if (words > 0) fr.st.store(a.states + i * words);
        a.code[i] = fr.code;
        if (a.hstep) a.hstep[i] = fr.hstep;
    }
}

struct ETune { int block, minb, unroll, lanes; };   // lanes: per orbit (1 = one orbit per thread)

typedef cudaError_t (*ELaunchFn)(const cl_run& run, const EArgs& a, int grid, const ETune& t, cudaStream_t st,
                                 LaunchInfo* info);

template <class Sys, typename Real, class F, int TAU_UNROLL, int MINB>
cudaError_t launch_ensemble_v(const cl_run& run, const EArgs& a, int grid, cudaStream_t st, LaunchInfo* info) {
    const Sys sys = SysMaker<Sys>::make(run, nullptr);
    auto k = ensemble_kernel<Sys, Real, F, TAU_UNROLL, MINB>;
    k<<<grid, 128, 0, st>>>(a, sys);
    cudaError_t e = cudaGetLastError();
    if (info) {
        cudaFuncAttributes at;
        if (cudaFuncGetAttributes(&at, k) == cudaSuccess) info->regs = at.numRegs;
        info->block = 128;
        info->grid = grid;
    }
    return e;
}

// Tunable variants: register cap (blocks per SM 1, 2, 4) x tau loop (runtime, or unrolled at the class's tau U).
template <class Sys, typename Real, class F, int U>
cudaError_t launch_ensemble(const cl_run& run, const EArgs& a, int grid, const ETune& t, cudaStream_t st,
                            LaunchInfo* info) {
    if (t.lanes > 1) return cudaErrorNotSupported;
    const bool unrolled = U > 1 && t.unroll == U && a.tau == U;
    if (unrolled) {
        if (t.minb == 1) return launch_ensemble_v<Sys, Real, F, U, 1>(run, a, grid, st, info);
        if (t.minb == 2) return launch_ensemble_v<Sys, Real, F, U, 2>(run, a, grid, st, info);
        if (t.minb == 4) return launch_ensemble_v<Sys, Real, F, U, 4>(run, a, grid, st, info);
    } else {
        if (t.minb == 1) return launch_ensemble_v<Sys, Real, F, 1, 1>(run, a, grid, st, info);
        if (t.minb == 2) return launch_ensemble_v<Sys, Real, F, 1, 2>(run, a, grid, st, info);
        if (t.minb == 4) return launch_ensemble_v<Sys, Real, F, 1, 4>(run, a, grid, st, info);
    }
    return cudaErrorInvalidValue;
}

void register_ensemble(const char* key, ELaunchFn fn);

struct ERegistrar {
    ERegistrar(const char* key, ELaunchFn fn) { register_ensemble(key, fn); }
};

}  // namespace cl
