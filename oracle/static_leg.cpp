// oracle/static_leg.cpp -- TEST INFRASTRUCTURE (the CPU oracle, statically sized). Only tests/ and the cpu_baseline
// / reference legs of bench.py load it; the product never does.
//
// The same restatement of the reference's per-orbit body as oracle_capi.cpp's run_orbit (src/Tangent/orbit.jl:44-60
// driven as `_orbit_kernel!` drives it, src/Tangent/propagate.jl:32-50), specialised at compile time on the tangent
// dimension D and the frame width K the way Julia specialises `_orbit_body` on SVector{D} / SMatrix{D, K}
// (StaticArrays.jl unrolls every fixed-size loop): each driver below is flattened, so every function of oracle.hpp it
// calls is inlined with its sizes as constants and the loops are unrolled. It executes the same operations in the
// same order as the runtime-sized oracle (no contraction, fma only where the reference writes it), so its records are
// bit for bit the oracle's; it exists to time the reference's CPU algorithm at its own speed. Map systems only
// (standard, wrapped standard, Froeschle, wrapped Froeschle), every frame of the run with the same K (a (GALI, SALI)
// chain carries its separate k = 2 SALI frame as the oracle does). Orbits run on a pool of std::threads taking
// chunks from an atomic counter.
#include <atomic>
#include <cstring>
#include <thread>
#include <vector>

#include "oracle.hpp"

using namespace orc;

namespace {

constexpr int8_t S_OK = 0, S_STATE = 1, S_W = 2, S_REDUCER = 3;   // orbit.jl:1

int64_t fbytes(const cl_frame& f) {
    int64_t b = 0;
    for (int r = 0; r < f.n_reducers; ++r) b += state_bytes_of(f.reducers[r], f.k);
    return b;
}

template <int S, int DK>
inline int8_t status_s(const double* x, const double* W) {   // _status, orbit.jl:3
    for (int i = 0; i < S; ++i) if (!isfin(x[i])) return S_STATE;
    for (int i = 0; i < DK; ++i) if (!isfin(W[i])) return S_W;
    return S_OK;
}

template <int MM, int SYS, int D, int S, int K>
__attribute__((flatten)) void orbit_static(const cl_run& run, int64_t i, const cl_buffers& b) {
    const int nf = run.n_frames;
    const int64_t n0 = run.n0;
    const int64_t steps = run.steps > 0 ? run.steps : run.N - n0;
    double x[S];
    double W[CL_MAX_FRAMES][D * K];
    double Ws[CL_MAX_FRAMES][D * 2];
    uint8_t st[CL_MAX_FRAMES][24 * CL_MAX_K + 32 + 72 + 16 * CL_MAX_K + 72];
    int64_t sb[CL_MAX_FRAMES];
    bool alive[CL_MAX_FRAMES];
    int8_t code[CL_MAX_FRAMES];
    int64_t hstep[CL_MAX_FRAMES];
    int sali_slot[CL_MAX_FRAMES];
    const double* xin = (n0 == 0 && b.x0) ? b.x0 : b.x;
    std::memcpy(x, xin + i * S, sizeof(double) * S);
    bool any = false;
    for (int f = 0; f < nf; ++f) {
        sb[f] = fbytes(run.frames[f]);
        std::memset(st[f], 0, sizeof st[f]);
        if (n0 == 0) {
            if (b.W0[f]) std::memcpy(W[f], b.W0[f] + i * D * K, sizeof(double) * D * K);
            else seeded_frame<MM>(run.seed, run.orbit_base + i + 1, D, K, W[f]);
            code[f] = S_OK;
            hstep[f] = 0;
            alive[f] = true;
        } else {
            std::memcpy(W[f], b.W[f] + i * D * K, sizeof(double) * D * K);
            if (sb[f]) std::memcpy(st[f], static_cast<const uint8_t*>(b.states[f]) + i * sb[f], sb[f]);
            code[f] = b.code[f][i];
            hstep[f] = b.hstep[f] ? b.hstep[f][i] : 0;
            alive[f] = code[f] == S_OK;
        }
        any = any || alive[f];
        sali_slot[f] = -1;
        const cl_frame& fr = run.frames[f];
        for (int r = 1; r < fr.n_reducers; ++r)
            if (fr.reducers[r].kind == CL_RED_SALI && fr.reducers[r - 1].kind == CL_RED_GALI && K > 2) sali_slot[f] = r;
        if (sali_slot[f] >= 0) std::memcpy(Ws[f], W[f], sizeof(double) * D * 2);
    }
    if (!any) return;
    int64_t n = n0;
    const int tau = run.tau;
    const int64_t handoffs = steps / tau;
    for (int64_t h = 0; h < handoffs; ++h) {
        for (int t = 0; t < tau; ++t) {
            double M[D * D];
            if constexpr (SYS == CL_SYS_STANDARD) Systems<MM>::standard(run.sys.K, x, M);
            else if constexpr (SYS == CL_SYS_WRAPPED_STANDARD) Systems<MM>::wrapped(run.sys.K, x, M);
            else if constexpr (SYS == CL_SYS_FROESCHLE) Systems<MM>::froeschle(run.sys.nu, run.sys.kappa, run.sys.mu, x, M);
            else Systems<MM>::wrapped_froeschle(run.sys.nu, run.sys.kappa, run.sys.mu, x, M);
            for (int f = 0; f < nf; ++f) {
                if (!alive[f]) continue;
                double Wn[D * K];
                fused_product(M, W[f], Wn, D, D, K);
                std::memcpy(W[f], Wn, sizeof(double) * D * K);
                if (sali_slot[f] >= 0) {
                    double Wm[D * 2];
                    fused_product(M, Ws[f], Wm, D, D, 2);
                    std::memcpy(Ws[f], Wm, sizeof(double) * D * 2);
                }
            }
        }
        n += tau;
        bool still = false;
        for (int f = 0; f < nf; ++f) {
            if (!alive[f]) continue;
            const cl_frame& fr = run.frames[f];
            const int8_t c = status_s<S, D * K>(x, W[f]);
            if (c != S_OK) { code[f] = c; hstep[f] = n; alive[f] = false; continue; }
            uint8_t* p = st[f];
            for (int r = 0; r < fr.n_reducers; ++r) {   // _apply (orbit.jl:23-28)
                if (r == sali_slot[f]) Reducers<MM>::step(fr.reducers[r], p, n, Ws[f], D, 2);
                else Reducers<MM>::step(fr.reducers[r], p, n, W[f], D, K);
                p += state_bytes_of(fr.reducers[r], K);
            }
            p = st[f];
            bool failed = false;
            for (int r = 0; r < fr.n_reducers; ++r) {
                failed = failed || Reducers<MM>::failed(fr.reducers[r], p, K);
                p += state_bytes_of(fr.reducers[r], K);
            }
            if (failed) { code[f] = S_REDUCER; hstep[f] = n; alive[f] = false; continue; }
            still = true;
        }
        if (!still) break;
    }
    for (int f = 0; f < nf; ++f)
        if (alive[f]) {   // orbit.jl:58: the final status check only at step N
            const int8_t c = status_s<S, D * K>(x, W[f]);
            code[f] = n == run.N ? c : S_OK;
            hstep[f] = n;
        }
    std::memcpy(b.x + i * S, x, sizeof(double) * S);
    for (int f = 0; f < nf; ++f) {
        if (n0 > 0 && b.code[f][i] != S_OK) continue;   // frozen since an earlier launch
        std::memcpy(b.W[f] + i * D * K, W[f], sizeof(double) * D * K);
        if (sb[f]) std::memcpy(static_cast<uint8_t*>(b.states[f]) + i * sb[f], st[f], sb[f]);
        b.code[f][i] = code[f];
        if (b.hstep[f]) b.hstep[f][i] = hstep[f];
    }
}

typedef void (*OrbitFn)(const cl_run&, int64_t, const cl_buffers&);

template <int MM>
OrbitFn pick(const cl_run& r) {
    const int k = r.frames[0].k;
    for (int f = 1; f < r.n_frames; ++f)
        if (r.frames[f].k != k) return nullptr;
    switch (r.sys.kind) {
        case CL_SYS_STANDARD:
            if (k == 1) return orbit_static<MM, CL_SYS_STANDARD, 2, 2, 1>;
            if (k == 2) return orbit_static<MM, CL_SYS_STANDARD, 2, 2, 2>;
            break;
        case CL_SYS_WRAPPED_STANDARD:
            if (k == 1) return orbit_static<MM, CL_SYS_WRAPPED_STANDARD, 2, 4, 1>;
            if (k == 2) return orbit_static<MM, CL_SYS_WRAPPED_STANDARD, 2, 4, 2>;
            break;
        case CL_SYS_FROESCHLE:
            if (k == 2) return orbit_static<MM, CL_SYS_FROESCHLE, 4, 4, 2>;
            if (k == 4) return orbit_static<MM, CL_SYS_FROESCHLE, 4, 4, 4>;
            break;
        case CL_SYS_WRAPPED_FROESCHLE:
            if (k == 2) return orbit_static<MM, CL_SYS_WRAPPED_FROESCHLE, 4, 8, 2>;
            if (k == 4) return orbit_static<MM, CL_SYS_WRAPPED_FROESCHLE, 4, 8, 4>;
            break;
        default: break;
    }
    return nullptr;
}

}  // namespace

extern "C" {

// 0 when the run is covered (map system, every frame of one K in the compiled set), else -3.
int oracle_static_supported(const cl_run* run) {
    if (!run || run->n_frames < 1) return -3;
    return pick<MATH_PORTABLE>(*run) ? 0 : -3;
}

// The statically sized oracle over n orbits (orbit-major host buffers, as oracle_propagate), portable math, on
// `threads` threads (<= 0: the hardware's count). Returns 0, or -3 for a run it does not cover.
int oracle_static_propagate(const cl_run* run, int64_t n, const cl_buffers* b, int threads) {
    if (!run || !b) return -1;
    const OrbitFn fn = pick<MATH_PORTABLE>(*run);
    if (!fn) return -3;
    const int hw = static_cast<int>(std::thread::hardware_concurrency());
    const int nt = threads > 0 ? threads : (hw > 0 ? hw : 1);
    std::atomic<int64_t> next{0};
    const int64_t chunk = 16;
    auto work = [&]() {
        for (;;) {
            const int64_t lo = next.fetch_add(chunk);
            if (lo >= n) return;
            const int64_t hi = lo + chunk < n ? lo + chunk : n;
            for (int64_t i = lo; i < hi; ++i) fn(*run, i, *b);
        }
    };
    std::vector<std::thread> pool;
    for (int t = 1; t < nt; ++t) pool.emplace_back(work);
    work();
    for (auto& t : pool) t.join();
    return 0;
}

}  // extern "C"
