// cl_shadow.cu -- the two-trajectory estimator (src/Lyapunov/two_trajectory.jl): per orbit a shadow started at
// distance d0 from the reference along a unit direction u0, both advanced by the map's `forward`, and every tau steps
// the separation d is measured, log(d / d_prev) added to a Neumaier sum and the shadow put back at distance d0 along
// the separation (Algorithm 1 to 3). One orbit per thread, the states in registers; a launch covers a window of
// steps and carries the end record, which is written in the isbits layout of the reference's `ShadowEnd{s, Float64}`
// (x, y, sum, dprev, code, step, value).
//
// `separation` and `displaced` (src/Lyapunov/separation.jl) are the plain difference and sum on lifted states, and
// for WrappedStandardMap the minimal image in (-pi, pi] and the reduction with carried winding counts.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <type_traits>
#include <vector>

#include "../../include/chaoslab_b200.h"
#include "cl_gauss.cuh"
#include "cl_hostcall.cuh"
#include "cl_split.cuh"

namespace cl {

int capi_fail(int code, const std::string& msg);      // cl_capi.cu
int capi_map_cuda(cudaError_t e, const char* where);  // cl_capi.cu
int capi_validate(const cl_run& r);                   // cl_capi.cu
void capi_count_launch();                             // cl_capi.cu

namespace {

struct ShArgs {
    i64 n, n0, steps, N;
    int tau;
    double d0;
    const double* x0;   // n x S (orbit-major)
    const double* u0;   // n x D, or NULL: the seeded direction (first column of the seeded frame)
    uint64_t* ends;     // n records of ShadowEnd{S, Float64}
    uint64_t seed;
    i64 orbit_base;
};

template <class Sys> struct Wrapped { static constexpr bool value = false; };
template <> struct Wrapped<SysWrapped> { static constexpr bool value = true; };

// separation (separation.jl:9, :25-28)
template <class Sys>
__device__ __forceinline__ void separation(const double* x, const double* y, double* delta) {
    constexpr int D = Sys::D;
    if constexpr (Wrapped<Sys>::value) {
        const double tp = 2 * jl_pi(), h = tp / 2;
#pragma unroll
        for (int i = 0; i < 2; ++i) {
            const double u = y[i] - x[i];
            delta[i] = u > h ? u - tp : (u <= -h ? u + tp : u);
        }
    } else {
#pragma unroll
        for (int i = 0; i < D; ++i) delta[i] = y[i] - x[i];
    }
}

// displaced (separation.jl:17, :30-35): y = x + delta; wrapped: reduce both coordinates, add the counts
template <class Sys>
__device__ __forceinline__ void displaced(const double* x, const double* delta, double* y) {
    constexpr int D = Sys::D;
    if constexpr (Wrapped<Sys>::value) {
        const double tp = 2 * jl_pi();
        double xr, a, pr, b;
        wrap_reduce(x[0] + delta[0], tp, xr, a);
        wrap_reduce(x[1] + delta[1], tp, pr, b);
        y[0] = xr; y[1] = pr; y[2] = x[2] + a; y[3] = x[3] + b;
    } else {
#pragma unroll
        for (int i = 0; i < D; ++i) y[i] = x[i] + delta[i];
    }
}

// forward (the map's own, without its tangent where the system separates them)
template <class Sys>
__device__ __forceinline__ void fwd(const Sys& sys, double* z) {
    if constexpr (std::is_same<Sys, SysSplitHH>::value) {
        SplitJac unused;
        sys.forward(z, unused);
    } else {
        typename Sys::Jac J;
        sys.jac(z, J);
        sys.forward(z, J);
    }
}

template <int S>
__device__ __forceinline__ void store_end(uint64_t* e, const double* x, const double* y, const CS& acc, double dprev,
                                          int8_t code, i64 step, double value) {
#pragma unroll
    for (int c = 0; c < S; ++c) { e[c] = __double_as_longlong(x[c]); e[S + c] = __double_as_longlong(y[c]); }
    e[2 * S] = __double_as_longlong(acc.s);
    e[2 * S + 1] = __double_as_longlong(acc.c);
    e[2 * S + 2] = __double_as_longlong(dprev);
    e[2 * S + 3] = static_cast<uint64_t>(static_cast<uint8_t>(code));
    e[2 * S + 4] = static_cast<uint64_t>(step);
    e[2 * S + 5] = __double_as_longlong(value);
}

// One orbit's end record in registers (ShadowEnd{S, Float64}).
template <class Sys>
struct ShadowOrbit {
    static constexpr int D = Sys::D, S = Sys::S, W = 2 * S + 6;
    double x[S], y[S];
    CS acc;
    double dprev;
    int8_t code;
    i64 step;
    double value;

    // _shadow_start (two_trajectory.jl:31-36): y = displaced(x0, d0 u0), its realised separation, a code
    __device__ __forceinline__ void start(const ShArgs& a, i64 i) {
        double delta[D], u[D];
#pragma unroll
        for (int c = 0; c < S; ++c) x[c] = a.x0[i * S + c];
        if (a.u0) {
#pragma unroll
            for (int c = 0; c < D; ++c) u[c] = a.u0[i * D + c];
        } else {
            seeded_frame<D, 1>(a.seed, a.orbit_base + i + 1, u);
        }
#pragma unroll
        for (int c = 0; c < D; ++c) delta[c] = a.d0 * u[c];
        displaced<Sys>(x, delta, y);
        separation<Sys>(x, y, delta);
        dprev = safe_norm<D>(delta);
        acc = CS{0.0, 0.0};
        code = !(isfin(dprev) && dprev > 0) ? 2 : (dprev < a.d0 / 2 || dprev > 2 * a.d0 ? 3 : 0);
        step = 0;
        value = dprev;
    }
    __device__ __forceinline__ void load(const uint64_t* e) {
#pragma unroll
        for (int c = 0; c < S; ++c) { x[c] = __longlong_as_double(e[c]); y[c] = __longlong_as_double(e[S + c]); }
        acc.s = __longlong_as_double(e[2 * S]);
        acc.c = __longlong_as_double(e[2 * S + 1]);
        dprev = __longlong_as_double(e[2 * S + 2]);
        code = static_cast<int8_t>(e[2 * S + 3] & 0xff);
        step = static_cast<i64>(e[2 * S + 4]);
        value = __longlong_as_double(e[2 * S + 5]);
    }
    __device__ __forceinline__ void store(uint64_t* e) const { store_end<S>(e, x, y, acc, dprev, code, step, value); }

    // _shadow_body (two_trajectory.jl:59-80) over `steps` steps from global step n; sets code / step / value
    __device__ __forceinline__ void body(const Sys& sys, i64 n, i64 steps, int tau, double d0) {
        double delta[D];
        for (i64 h = 0; h < steps / tau; ++h) {
            for (int t = 0; t < tau; ++t) {
                fwd(sys, x);
                fwd(sys, y);
            }
            n += tau;
            bool fin = true;
            double bad = 0.0;
#pragma unroll
            for (int c = S - 1; c >= 0; --c) if (!isfin(y[c])) { fin = false; bad = y[c]; }
#pragma unroll
            for (int c = S - 1; c >= 0; --c) if (!isfin(x[c])) { fin = false; bad = x[c]; }
            if (!fin) { code = 1; step = n; value = bad; return; }
            separation<Sys>(x, y, delta);
            const double d = safe_norm<D>(delta);
            if (!(isfin(d) && d > 0)) { code = 2; step = n; value = d; return; }
            cs_add(acc, cl_log(d / dprev));
            const double f = d0 / d;
#pragma unroll
            for (int c = 0; c < D; ++c) delta[c] = delta[c] * f;
            displaced<Sys>(x, delta, y);
            separation<Sys>(x, y, delta);
            dprev = safe_norm<D>(delta);
            if (!(dprev >= d0 / 2 && dprev <= 2 * d0)) {
                code = (isfin(dprev) && dprev > 0) ? 3 : 2;
                step = n;
                value = dprev;
                return;
            }
        }
        code = 0;
        step = n;
        value = dprev;
    }
};

// One launch window of one orbit (the estimator: _shadow_kernel!, two_trajectory.jl:108-115)
template <class Sys>
__global__ void __launch_bounds__(128) shadow_kernel(const ShArgs a, const Sys sys) {
    using O = ShadowOrbit<Sys>;
    const i64 i = static_cast<i64>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= a.n) return;
    uint64_t* e = a.ends + i * O::W;
    O o;
    if (a.n0 == 0) {
        o.start(a, i);
        if (o.code != 0) { o.store(e); return; }
    } else {
        o.load(e);
        if (o.code != 0) return;   // failed in an earlier launch: frozen
    }
    o.body(sys, a.n0, a.steps, a.tau, a.d0);
    o.store(e);
}

// The recorder's two-trajectory method (_shadow_record_kernel!, src/Experiments/run_device.jl:80-100): segments
// between the grid steps of the window; row g of R[col, g, orbit] (1 + 7 + S columns) gets X2 so far in column 1
// and the reference state in the state columns; a failure stores its 1-based grid index in fail[orbit].
template <class Sys>
__global__ void __launch_bounds__(128) shadow_record_kernel(const ShArgs a, const Sys sys, const i64* grid, int n_grid,
                                                            double* R, i64* fail) {
    using O = ShadowOrbit<Sys>;
    constexpr int S = O::S, NCOL = 1 + 7 + S;
    const i64 i = static_cast<i64>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= a.n) return;
    uint64_t* e = a.ends + i * O::W;
    O o;
    if (a.n0 == 0) {
        o.start(a, i);
        // _blank_end: the start is made in the first segment; a bad start fails that segment
    } else {
        o.load(e);
        if (o.code != 0) return;
    }
    int glo = 0;
    while (glo < n_grid && grid[glo] <= a.n0) ++glo;
    int ghi = glo - 1;
    while (ghi + 1 < n_grid && grid[ghi + 1] <= a.n0 + a.steps) ++ghi;
    i64 n = a.n0;
    double* Ri = R + i * static_cast<i64>(NCOL) * n_grid;
    for (int g = glo; g <= ghi; ++g) {
        const i64 target = grid[g];
        if (o.code == 0) o.body(sys, n, target - n, a.tau, a.d0);
        if (o.code != 0) { fail[i] = g + 1; o.store(e); return; }
        n = target;
        double* row = Ri + static_cast<i64>(g) * NCOL;
        row[0] = cs_total(o.acc) / static_cast<double>(target);
#pragma unroll
        for (int j = 0; j < S; ++j) row[8 + j] = o.x[j];
    }
    if (o.code == 0 && n < a.n0 + a.steps) {
        o.body(sys, n, a.n0 + a.steps - n, a.tau, a.d0);
        if (o.code != 0) fail[i] = ghi + 2;
    } else if (o.code != 0 && glo > ghi) {
        fail[i] = ghi + 2;   // a bad start in a window with no grid step
    }
    o.store(e);
}

struct RecOut { const i64* grid; int n_grid; double* R; i64* fail; };   // grid records (NULL grid: none)

typedef cudaError_t (*ShadowFn)(const cl_run& run, const ShArgs& a, const RecOut& r, cudaStream_t st);

template <class Sys>
cudaError_t launch_shadow(const cl_run& run, const ShArgs& a, const RecOut& r, cudaStream_t st) {
    const Sys sys = SysMaker<Sys>::make(run, nullptr);
    const unsigned grid = static_cast<unsigned>((a.n + 127) / 128);
    if (r.grid) shadow_record_kernel<Sys><<<grid, 128, 0, st>>>(a, sys, r.grid, r.n_grid, r.R, r.fail);
    else shadow_kernel<Sys><<<grid, 128, 0, st>>>(a, sys);
    return cudaGetLastError();
}

ShadowFn shadow_fn(const cl_run& r) {
    switch (r.sys.kind) {
        case CL_SYS_STANDARD: return launch_shadow<SysStandard>;
        case CL_SYS_WRAPPED_STANDARD: return launch_shadow<SysWrapped>;
        case CL_SYS_FROESCHLE: return launch_shadow<SysFroeschle>;
        case CL_SYS_HH_GAUSS: return launch_shadow<SysGauss3HH>;
        case CL_SYS_HH_SPLIT: return launch_shadow<SysSplitHH>;
        case CL_SYS_LINEAR:
            if (r.d == 2) return launch_shadow<SysLinear<2>>;
            if (r.d == 4) return launch_shadow<SysLinear<4>>;
            if (r.d == 6) return launch_shadow<SysLinear<6>>;
            return nullptr;
        case CL_SYS_CHAIN:
            switch (r.sys.n_sites) {
                case 2: return launch_shadow<SysChain<2>>;
                case 3: return launch_shadow<SysChain<3>>;
                case 4: return launch_shadow<SysChain<4>>;
                case 5: return launch_shadow<SysChain<5>>;
                case 6: return launch_shadow<SysChain<6>>;
                case 7: return launch_shadow<SysChain<7>>;
                case 8: return launch_shadow<SysChain<8>>;
            }
            return nullptr;
    }
    return nullptr;
}

// The run's checks (system, tau, N, launch window) through propagate's validation with a placeholder frame.
int check_shadow(const cl_run& run, double d0, ShadowFn* fn) {
    cl_run r = run;
    r.n_frames = 1;
    std::memset(&r.frames[0], 0, sizeof r.frames[0]);
    r.frames[0].k = 1;
    r.precision = CL_PREC_FP64;
    const int v = capi_validate(r);
    if (v) return v;
    if (!(std::isfinite(d0) && d0 > 0)) return capi_fail(CL_EINVAL, "d0 must be finite and positive");
    *fn = shadow_fn(run);
    if (!*fn) return capi_fail(CL_EUNSUPPORTED, "no compiled two-trajectory kernel for this system");
    return 0;
}

ShArgs shargs(const cl_run& run, int64_t n, const double* x0, const double* u0, void* ends, double d0, int64_t n0,
              int64_t steps) {
    ShArgs a;
    a.n = n; a.n0 = n0; a.steps = steps; a.N = run.N; a.tau = run.tau; a.d0 = d0;
    a.x0 = x0; a.u0 = u0; a.ends = static_cast<uint64_t*>(ends);
    a.seed = run.seed; a.orbit_base = run.orbit_base;
    return a;
}

}  // namespace
}  // namespace cl

using namespace cl;

extern "C" {

int64_t cl_b200_shadow_bytes(int32_t s) { return s > 0 ? 8 * (2 * static_cast<int64_t>(s) + 6) : -1; }

int cl_b200_shadow_device(const cl_run* run, int64_t n, const double* x0, const double* u0, void* ends, double d0,
                          void* stream) {
    if (!run || n <= 0 || !ends || (run->n0 == 0 && !x0)) return capi_fail(CL_EINVAL, "bad arguments");
    ShadowFn fn;
    const int v = check_shadow(*run, d0, &fn);
    if (v) return v;
    const int64_t steps = run->steps > 0 ? run->steps : run->N - run->n0;
    const cudaError_t e = fn(*run, shargs(*run, n, x0, u0, ends, d0, run->n0, steps), RecOut{nullptr, 0, nullptr, nullptr},
                             static_cast<cudaStream_t>(stream));
    capi_count_launch();
    return e == cudaSuccess ? 0 : capi_map_cuda(e, "two-trajectory launch");
}

int cl_b200_shadow_record_device(const cl_run* run, int64_t n, const double* x0, const double* u0, void* ends,
                                 double d0, const int64_t* grid, int32_t n_grid, double* R, int64_t* fail,
                                 void* stream) {
    if (!run || n <= 0 || !ends || (run->n0 == 0 && !x0) || !grid || n_grid < 1 || !R || !fail)
        return capi_fail(CL_EINVAL, "bad arguments");
    ShadowFn fn;
    const int v = check_shadow(*run, d0, &fn);
    if (v) return v;
    const int64_t steps = run->steps > 0 ? run->steps : run->N - run->n0;
    const cudaError_t e = fn(*run, shargs(*run, n, x0, u0, ends, d0, run->n0, steps),
                             RecOut{reinterpret_cast<const i64*>(grid), n_grid, R, reinterpret_cast<i64*>(fail)},
                             static_cast<cudaStream_t>(stream));
    capi_count_launch();
    return e == cudaSuccess ? 0 : capi_map_cuda(e, "two-trajectory record launch");
}

// Host buffers: copies in, windows of run.steps steps from run.n0 to run.N, copies out; with `grid`, the records.
static int shadow_host(const cl_run* run, int64_t n, const double* x0, const double* u0, void* ends, double d0,
                       const int64_t* grid, int32_t n_grid, double* R, int64_t* fail, cl_prov* prov) {
    if (!run || n <= 0 || !x0 || !ends || (grid && (n_grid < 1 || !R || !fail))) return capi_fail(CL_EINVAL, "bad arguments");
    ShadowFn fn;
    int rc = check_shadow(*run, d0, &fn);
    if (rc) return rc;
    const int S = run->s, D = run->d, ncol = 1 + 7 + S;
    std::vector<HostArray> arr = {
        {const_cast<double*>(x0), sizeof(double) * S * n, false, nullptr},
        {const_cast<double*>(u0), sizeof(double) * D * n, false, nullptr},
        {ends, static_cast<size_t>(cl_b200_shadow_bytes(S)) * n, true, nullptr},
        {const_cast<int64_t*>(grid), grid ? sizeof(int64_t) * n_grid : 0, false, nullptr},
        {grid ? R : nullptr, grid ? sizeof(double) * ncol * n_grid * n : 0, true, nullptr},
        {grid ? fail : nullptr, grid ? sizeof(int64_t) * n : 0, true, nullptr}};
    rc = host_windows(*run, arr, [&](const cl_run& w, cudaStream_t st) {
        const cudaError_t e = fn(w, shargs(w, n, static_cast<double*>(arr[0].dev), static_cast<double*>(arr[1].dev),
                                           arr[2].dev, d0, w.n0, w.steps),
                                 RecOut{static_cast<const i64*>(arr[3].dev), n_grid, static_cast<double*>(arr[4].dev),
                                        static_cast<i64*>(arr[5].dev)}, st);
        capi_count_launch();
        return e == cudaSuccess ? 0 : capi_map_cuda(e, "two-trajectory launch");
    }, prov, "two-trajectory");
    if (rc == 0 && prov)
        std::snprintf(prov->variant, sizeof prov->variant, "two-trajectory s%d d%d%s", S, D, grid ? " records" : "");
    return rc;
}

int cl_b200_shadow(const cl_run* run, int64_t n, const double* x0, const double* u0, void* ends, double d0,
                   cl_prov* prov) {
    return shadow_host(run, n, x0, u0, ends, d0, nullptr, 0, nullptr, nullptr, prov);
}

int cl_b200_shadow_record(const cl_run* run, int64_t n, const double* x0, const double* u0, void* ends, double d0,
                          const int64_t* grid, int32_t n_grid, double* R, int64_t* fail, cl_prov* prov) {
    if (!grid) return capi_fail(CL_EINVAL, "bad arguments");
    return shadow_host(run, n, x0, u0, ends, d0, grid, n_grid, R, fail, prov);
}

}  // extern "C"
