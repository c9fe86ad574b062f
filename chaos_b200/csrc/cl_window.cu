// cl_window.cu -- the indicator recorder's window kinds on the device (src/Experiments/run_indicator_device.jl:62-91):
// the orbit advanced one handoff at a time with the deviation column reset to (1, 0) at each handoff (it is never
// read), the chain (RunMonitor, reader) with one reader reducer:
//   WeightedPhaseAdvance (src/Indicators/naff_reducer.jl:122-243): the weighted mean phase advance of a planar or a
//     lifted-angle observable over H horizons, two windows each, Neumaier sums A = sum w Delta and B = sum w;
//   WeightedBirkhoff (src/Indicators/wbirkhoff_reducer.jl:18-110, wbirkhoff.jl:78-90): the weighted Birkhoff
//     averages of K observables over H horizons, the running maximum |f|;
// both with the weight birkhoff_weight(min(j, N - j) / N, p) = exp(-1 / (t^p (1 - t)^p)) (naff_reducer.jl:13-17).
// At every grid step the row det_max, symp_max, M_max, x[0 .. ns-1]; the tables are the reader's reducer_final on the
// host. States (MonState, then the reader's isbits state in Julia's layout) are carried in place across launches.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/chaoslab_b200.h"
#include "cl_hostcall.cuh"
#include "cl_monitor.cuh"
#include "cl_registry.cuh"

namespace cl {

int capi_fail(int code, const std::string& msg);      // cl_capi.cu
int capi_map_cuda(cudaError_t e, const char* where);  // cl_capi.cu
int capi_validate(const cl_run& r);                   // cl_capi.cu
void capi_count_launch();                             // cl_capi.cu

namespace {

constexpr int kMaxReaderWords = (16 + CL_MAX_WINDOWS * (16 + 40 * CL_MAX_OBSERVABLES)) / 8;

struct WinArgs {
    i64 n, n0, steps, N;
    int tau, ns;
    double* x;
    uint64_t* states;     // MonState, then the reader's state
    int8_t* code;
    i64* hstep;
    const i64* grid;
    int n_grid, ncol;
    double* R;
    i64* fail;
    int kind, H, K, p, words;
    i64 win[CL_MAX_WINDOWS], maxwin;
    int ok[CL_MAX_OBSERVABLES], oa[CL_MAX_OBSERVABLES], ob[CL_MAX_OBSERVABLES];   // kinds, 0-based a, b (b raw)
};

// Julia's x^n for Float64 and n = 1..4 (power by squaring with the error terms carried, Base.Math): n = 1, 2, 3 are
// x, x x, (x x) x; n = 4 is the square of the square with the two product errors folded in.
__device__ __forceinline__ double jl_powi(double x, int n) {
    if (n == 1) return x;
    if (n == 2) return x * x;
    if (n == 3) return x * x * x;
    const double x2 = x * x, e2 = fma(x, x, -x2);
    const double err = (x2 * 2) * e2;
    const double x4 = x2 * x2, e4 = fma(x2, x2, -x4);
    return x4 + (e4 + err);
}

// _wb (naff_reducer.jl:13-17): the weight of sample j of a window of N at the mirrored argument
__device__ __forceinline__ double wb_weight(i64 j, i64 N, int p) {
    const double t = static_cast<double>(j < N - j ? j : N - j) / static_cast<double>(N);
    if (t <= 0.0 || t >= 1.0) return 0.0;
    return cl_exp(-1.0 / (jl_powi(t, p) * jl_powi(1.0 - t, p)));
}

// Typed fields of a state held as 8-byte words, at byte offsets of Julia's isbits layout
template <typename T> __device__ __forceinline__ T ld(const uint64_t* base, int byte) {
    T v;
    memcpy(&v, reinterpret_cast<const unsigned char*>(base) + byte, sizeof(T));
    return v;
}
template <typename T> __device__ __forceinline__ void sto(uint64_t* base, int byte, T v) {
    memcpy(reinterpret_cast<unsigned char*>(base) + byte, &v, sizeof(T));
}

// _unit_scale (naff_reducer.jl:36-41): the pair scaled by 2^-e, e the binary exponent of the larger magnitude
__device__ __forceinline__ void unit_scale(double& re, double& im) {
    const double m = jl_max(fabs(re), fabs(im));
    int e = 0;
    if (isfinite(m) && m > 0) {
        e = static_cast<int>((static_cast<unsigned long long>(__double_as_longlong(m)) >> 52) & 0x7ff) - 1023;
        e = e < -1000 ? -1000 : (e > 1000 ? 1000 : e);
    }
    const double s = cl_pow2(-e);
    re = re * s;
    im = im * s;
}

// _phase_inc (naff_reducer.jl:45-53): the principal argument of z / zp, NaN if either is exactly 0
__device__ __forceinline__ double phase_inc(double pr, double pi_, double zr, double zi) {
    if ((pr == 0.0 && pi_ == 0.0) || (zr == 0.0 && zi == 0.0)) return __longlong_as_double(0x7ff8000000000000LL);
    double wr = pr, wi = -pi_;   // conj(zp)
    double rr = zr * wr - zi * wi, ri = zr * wi + zi * wr;
    const double s = jl_max(fabs(rr), fabs(ri));
    if (!(s > 1e-280 && s < 1e280)) {
        unit_scale(zr, zi);
        unit_scale(pr, pi_);
        wr = pr; wi = -pi_;
        rr = zr * wr - zi * wi;
        ri = zr * wi + zi * wr;
    }
    return cl_atan2(ri, rr);
}

// WPAState{Float64, H} (naff_reducer.jl:160-167): hor[h] = (A1, B1, A2, B2) at 64 h; prev1, prev2, n, handoffs
// (Int32), nwrap (Int16), code (Int8) after the H horizons.
__device__ __forceinline__ void wpa_step(const WinArgs& a, uint64_t* st, i64 n, const double* x) {
    const int tail = 64 * a.H;
    if (ld<int8_t>(st, tail + 30) != 0) return;
    const int kind = a.ok[0];
    const double s1 = x[a.oa[0]], s2 = kind == CL_OBS_PLANAR ? x[a.ob[0] - 1] : (a.ob[0] == 0 ? 0.0 : x[a.ob[0] - 1]);
    if (!(isfinite(s1) && isfinite(s2))) {
        sto<i64>(st, tail + 16, n);
        sto<int8_t>(st, tail + 30, 1);
        return;
    }
    const int32_t s = ld<int32_t>(st, tail + 24);
    const int32_t h1 = s < 2147483647 ? s + 1 : s;
    if (s == 0) {
        sto<double>(st, tail, s1); sto<double>(st, tail + 8, s2);
        sto<i64>(st, tail + 16, n); sto<int32_t>(st, tail + 24, h1);
        return;
    }
    const double p1 = ld<double>(st, tail), p2 = ld<double>(st, tail + 8);
    const double pi_ = 3.141592653589793;
    const double d = kind == CL_OBS_PLANAR ? phase_inc(p1, p2, s1, s2) : (s1 - p1) + (2 * pi_) * (s2 - p2);
    const i64 j = s - 1;
    for (int h = 0; h < a.H; ++h) {   // _advance (naff_reducer.jl:176-186) with _accumulate (:66)
        const i64 N = a.win[h];
        if (j >= 2 * N) continue;
        const int off = 64 * h + (j < N ? 0 : 32);
        const double w = wb_weight(j < N ? j : j - N, N, a.p);
        if (w == 0.0) continue;
        CS A{ld<double>(st, off), ld<double>(st, off + 8)}, B{ld<double>(st, off + 16), ld<double>(st, off + 24)};
        cs_add(A, w * d);
        cs_add(B, w);
        sto<double>(st, off, A.s); sto<double>(st, off + 8, A.c);
        sto<double>(st, off + 16, B.s); sto<double>(st, off + 24, B.c);
    }
    const int16_t nw = ld<int16_t>(st, tail + 28);
    const bool flagged = kind == CL_OBS_PLANAR && fabs(d) > (9.0 * pi_) / 10.0 && s <= 2 * a.maxwin && nw < 32767;
    sto<double>(st, tail, s1); sto<double>(st, tail + 8, s2);
    sto<i64>(st, tail + 16, n); sto<int32_t>(st, tail + 24, h1);
    if (flagged) sto<int16_t>(st, tail + 28, static_cast<int16_t>(nw + 1));
}

// The value of observable k of a Birkhoff reader at the orbit point (wbirkhoff.jl:51-56, run_indicator_chain.jl:23)
__device__ __forceinline__ double observable(const WinArgs& a, int k, const double* x) {
    switch (a.ok[k]) {
        case CL_OBS_COS: return cl_cos(static_cast<double>(a.ob[k]) * x[a.oa[k]]);
        case CL_OBS_SIN: return cl_sin(static_cast<double>(a.ob[k]) * x[a.oa[k]]);
        case CL_OBS_LIFTED: return x[a.oa[k]] + (2 * 3.141592653589793) * x[a.ob[k] - 1];
        default: return x[a.oa[k]];
    }
}

// WBState{Float64, H, K} (wbirkhoff_reducer.jl:40-52): hor[h] = (B, cells[k] = (A1, A2, S)) at h (16 + 40 K); n,
// handoffs (Int32), code (Int16) after the H horizons.
__device__ __forceinline__ void wb_step(const WinArgs& a, uint64_t* st, i64 n, const double* x) {
    const int hb = 16 + 40 * a.K, tail = a.H * hb;
    if (ld<int16_t>(st, tail + 12) != 0) return;
    const int32_t hand = ld<int32_t>(st, tail + 8);
    if (static_cast<i64>(hand) >= 2 * a.maxwin) {   // every horizon frozen: only the counters advance
        sto<i64>(st, tail, n);
        if (hand < 2147483647) sto<int32_t>(st, tail + 8, hand + 1);
        return;
    }
    double v[CL_MAX_OBSERVABLES];
    int bad = 0;
    for (int k = 0; k < a.K; ++k) {
        v[k] = observable(a, k, x);
        if (bad == 0 && !isfinite(v[k])) bad = k + 1;
    }
    if (bad) {
        sto<i64>(st, tail, n);
        sto<int16_t>(st, tail + 12, static_cast<int16_t>(bad));
        return;
    }
    const i64 j = hand;
    for (int h = 0; h < a.H; ++h) {   // _wb_advance (wbirkhoff_reducer.jl:56-62) with _wb_sample (wbirkhoff.jl:86-90)
        const i64 N = a.win[h];
        if (j >= 2 * N) continue;
        const int i = j >= N ? 1 : 0;
        const double w = wb_weight(j - i * N, N, a.p);
        const int off = h * hb;
        if (i == 0 && w != 0.0) {
            CS B{ld<double>(st, off), ld<double>(st, off + 8)};
            cs_add(B, w);
            sto<double>(st, off, B.s); sto<double>(st, off + 8, B.c);
        }
        for (int k = 0; k < a.K; ++k) {
            const int c = off + 16 + 40 * k;
            sto<double>(st, c + 32, jl_max(ld<double>(st, c + 32), fabs(v[k])));
            if (w == 0.0) continue;
            const int ai = c + 16 * i;
            CS A{ld<double>(st, ai), ld<double>(st, ai + 8)};
            cs_add(A, w * v[k]);
            sto<double>(st, ai, A.s); sto<double>(st, ai + 8, A.c);
        }
    }
    sto<i64>(st, tail, n);
    sto<int32_t>(st, tail + 8, j < 2147483647 ? static_cast<int32_t>(j + 1) : hand);
}

__device__ __forceinline__ bool reader_failed(const WinArgs& a, uint64_t* st) {
    return a.kind == CL_WIN_PHASE_ADVANCE ? ld<int8_t>(st, 64 * a.H + 30) != 0
                                          : ld<int16_t>(st, a.H * (16 + 40 * a.K) + 12) != 0;
}

template <class Sys>
__global__ void __launch_bounds__(128) ind_window_kernel(const WinArgs a, const Sys sys) {
    constexpr int D = Sys::D, S = Sys::S;
    const i64 i = static_cast<i64>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= a.n) return;
    if (!(a.n0 == 0 || a.code[i] == STATUS_OK)) return;
    double x[S];
#pragma unroll
    for (int c = 0; c < S; ++c) x[c] = a.x[i * S + c];
    uint64_t* gst = a.states + i * (3 + a.words);
    MonState mon;
    uint64_t rs[kMaxReaderWords];
    if (a.n0 == 0) {
        mon.det_max = mon.symp_max = mon.M_max = 0.0;
        for (int w = 0; w < a.words; ++w) rs[w] = 0ull;
    } else {
        mon.det_max = __longlong_as_double(static_cast<long long>(gst[0]));
        mon.symp_max = __longlong_as_double(static_cast<long long>(gst[1]));
        mon.M_max = __longlong_as_double(static_cast<long long>(gst[2]));
        for (int w = 0; w < a.words; ++w) rs[w] = gst[3 + w];
    }
    int g = 0;
    while (g < a.n_grid && a.grid[g] <= a.n0) ++g;
    int ghi = g - 1;
    while (ghi + 1 < a.n_grid && a.grid[ghi + 1] <= a.n0 + a.steps) ++ghi;
    double* Ri = a.R + i * static_cast<i64>(a.ncol) * a.n_grid;
    i64 n = a.n0, h = a.n0;
    int8_t c = STATUS_OK;
    for (i64 hh = 0; hh < a.steps / a.tau; ++hh) {
        double W[D];   // the constant deviation column (1, 0)
        W[0] = 1.0;
#pragma unroll
        for (int l = 1; l < D; ++l) W[l] = 0.0;
        for (int t = 0; t < a.tau; ++t) {
            typename Sys::Jac J;
            sys.jac(x, J);
            sys.template apply<1>(J, W);
            sys.forward(x, J);
        }
        const i64 nn = n + a.tau;
        c = all_finite_x<D, S>(x) ? (all_finite<D>(W) ? STATUS_OK : STATUS_W) : STATUS_STATE;
        if (c == STATUS_OK) {
            monitor_step(sys, x, mon);
            if (a.kind == CL_WIN_PHASE_ADVANCE) wpa_step(a, rs, nn, x);
            else wb_step(a, rs, nn, x);
            if (reader_failed(a, rs)) c = STATUS_REDUCER;
        }
        h = nn;
        if (c != STATUS_OK) {
            a.fail[i] = (g <= ghi ? g : ghi + 1) + 1;
            break;
        }
        n = nn;
        if (g <= ghi && n == a.grid[g]) {
            double* row = Ri + static_cast<i64>(g) * a.ncol;
            row[0] = mon.det_max;
            row[1] = mon.symp_max;
            row[2] = mon.M_max;
#pragma unroll
            for (int j = 0; j < S; ++j)
                if (j < a.ns) row[3 + j] = x[j];
            ++g;
        }
    }
#pragma unroll
    for (int k = 0; k < S; ++k) a.x[i * S + k] = x[k];
    gst[0] = static_cast<uint64_t>(__double_as_longlong(mon.det_max));
    gst[1] = static_cast<uint64_t>(__double_as_longlong(mon.symp_max));
    gst[2] = static_cast<uint64_t>(__double_as_longlong(mon.M_max));
    for (int w = 0; w < a.words; ++w) gst[3 + w] = rs[w];
    a.code[i] = c;
    if (a.hstep) a.hstep[i] = h;
}

template <class Sys>
cudaError_t launch_window(const cl_run& run, const WinArgs& a, cudaStream_t st) {
    const Sys sys = SysMaker<Sys>::make(run, nullptr);
    ind_window_kernel<Sys><<<static_cast<unsigned>((a.n + 127) / 128), 128, 0, st>>>(a, sys);
    return cudaGetLastError();
}

int64_t reader_bytes(const cl_window& w) {
    return w.kind == CL_WIN_PHASE_ADVANCE ? 64 * static_cast<int64_t>(w.n_windows) + 32
                                          : 16 + static_cast<int64_t>(w.n_windows) * (16 + 40 * w.n_observables);
}

// The reader's constructor and check_run checks (naff_reducer.jl:150-154,236-243; wbirkhoff_reducer.jl:27-33,
// 118-135) that the kernel relies on, and the observable indices against the orbit point.
int check_window(const cl_run& r, const cl_window* w) {
    if (!w) return capi_fail(CL_EINVAL, "window is NULL");
    if (w->kind != CL_WIN_PHASE_ADVANCE && w->kind != CL_WIN_BIRKHOFF) return capi_fail(CL_EINVAL, "unknown window kind");
    if (w->n_windows < 1 || w->n_windows > CL_MAX_WINDOWS) return capi_fail(CL_EINVAL, "window: 1 to 4 horizons");
    for (int h = 0; h < w->n_windows; ++h)
        if (w->window[h] < 16) return capi_fail(CL_EINVAL, "window must be at least 16");
    if (w->birkhoff_order < 1 || w->birkhoff_order > 4) return capi_fail(CL_EINVAL, "birkhoff_order must be an integer from 1 to 4");
    const int K = w->n_observables;
    if (w->kind == CL_WIN_PHASE_ADVANCE ? K != 1 : (K < 1 || K > CL_MAX_OBSERVABLES))
        return capi_fail(CL_EINVAL, "observables: one for the phase advance, 1 to 8 for Birkhoff");
    for (int k = 0; k < K; ++k) {
        const int kind = w->obs_kind[k], ia = w->obs_a[k], ib = w->obs_b[k];
        const bool pa = kind == CL_OBS_PLANAR || kind == CL_OBS_LIFTED_ANGLE;
        if (pa != (w->kind == CL_WIN_PHASE_ADVANCE) || kind < CL_OBS_PLANAR || kind > CL_OBS_COORDINATE)
            return capi_fail(CL_EINVAL, "observable kind does not match the reader");
        if (ia < 1 || ia > r.s) return capi_fail(CL_EINVAL, "observable index outside the orbit point");
        const bool second = kind == CL_OBS_PLANAR || kind == CL_OBS_LIFTED || (kind == CL_OBS_LIFTED_ANGLE && ib != 0);
        if (second && (ib < 1 || ib > r.s)) return capi_fail(CL_EINVAL, "observable index outside the orbit point");
    }
    return 0;
}

int window_device(const cl_run* run, const cl_window* win, int64_t n, int32_t ns, double* x, void* states,
                  int8_t* code, int64_t* hstep, const int64_t* grid, int32_t n_grid, double* R, int64_t* fail,
                  void* stream) {
    if (!run || n <= 0 || !x || !states || !code || !grid || n_grid < 1 || !R || !fail || ns < 0)
        return capi_fail(CL_EINVAL, "bad arguments");
    int v = capi_validate(*run);
    if (v) return v;
    v = check_window(*run, win);
    if (v) return v;
    if (ns > run->s) return capi_fail(CL_EINVAL, "ns exceeds the state length");
    if (run->n_frames != 1 || run->frames[0].k != 1 || run->frames[0].n_reducers != 0 || run->precision != CL_PREC_FP64)
        return capi_fail(CL_EINVAL, "a window kind runs one frame with k = 1 and no reducers (the reader is the window)");
    WinArgs a;
    std::memset(&a, 0, sizeof a);
    a.n = n; a.n0 = run->n0; a.steps = run->steps > 0 ? run->steps : run->N - run->n0; a.N = run->N; a.tau = run->tau;
    a.ns = ns; a.x = x; a.states = static_cast<uint64_t*>(states); a.code = code;
    a.hstep = reinterpret_cast<i64*>(hstep); a.grid = reinterpret_cast<const i64*>(grid); a.n_grid = n_grid;
    a.ncol = 3 + ns; a.R = R; a.fail = reinterpret_cast<i64*>(fail);
    a.kind = win->kind; a.H = win->n_windows; a.K = win->n_observables; a.p = win->birkhoff_order;
    a.words = static_cast<int>(reader_bytes(*win) / 8);
    for (int h = 0; h < a.H; ++h) { a.win[h] = win->window[h]; a.maxwin = std::max<i64>(a.maxwin, win->window[h]); }
    for (int k = 0; k < a.K; ++k) { a.ok[k] = win->obs_kind[k]; a.oa[k] = win->obs_a[k] - 1; a.ob[k] = win->obs_b[k]; }
    cudaError_t err;
    switch (run->sys.kind) {
        case CL_SYS_STANDARD: err = launch_window<SysStandard>(*run, a, static_cast<cudaStream_t>(stream)); break;
        case CL_SYS_WRAPPED_STANDARD: err = launch_window<SysWrapped>(*run, a, static_cast<cudaStream_t>(stream)); break;
        case CL_SYS_LINEAR:
            if (run->d != 2) return capi_fail(CL_EUNSUPPORTED, "the window kinds cover 2 x 2 linear maps");
            err = launch_window<SysLinear<2>>(*run, a, static_cast<cudaStream_t>(stream));
            break;
        default: return capi_fail(CL_EUNSUPPORTED, "the window kinds cover the standard maps and 2 x 2 linear maps");
    }
    capi_count_launch();
    return err == cudaSuccess ? 0 : capi_map_cuda(err, "window launch");
}

}  // namespace
}  // namespace cl

using namespace cl;

extern "C" {

int64_t cl_b200_window_state_bytes(const cl_window* win) { return win ? reader_bytes(*win) : -1; }

int cl_b200_indicator_window_device(const cl_run* run, const cl_window* win, int64_t n, int32_t ns, double* x,
                                    void* states, int8_t* code, int64_t* hstep, const int64_t* grid, int32_t n_grid,
                                    double* R, int64_t* fail, void* stream) {
    return window_device(run, win, n, ns, x, states, code, hstep, grid, n_grid, R, fail, stream);
}

int cl_b200_indicator_window(const cl_run* run, const cl_window* win, int64_t n, int32_t ns, double* x, void* states,
                             int8_t* code, int64_t* hstep, const int64_t* grid, int32_t n_grid, double* R,
                             int64_t* fail, cl_prov* prov) {
    if (!run || n <= 0 || !x || !states || !code || !grid || n_grid < 1 || !R || !fail || ns < 0)
        return capi_fail(CL_EINVAL, "bad arguments");
    int rc = capi_validate(*run);
    if (rc) return rc;
    rc = check_window(*run, win);
    if (rc) return rc;
    const int s = run->s, ncol = 3 + ns;
    std::vector<HostArray> arr = {
        {x, sizeof(double) * s * n, true, nullptr},
        {states, static_cast<size_t>((24 + reader_bytes(*win)) * n), true, nullptr},
        {code, static_cast<size_t>(n), true, nullptr},
        {hstep, sizeof(int64_t) * n, true, nullptr},
        {const_cast<int64_t*>(grid), sizeof(int64_t) * n_grid, false, nullptr},
        {R, sizeof(double) * ncol * n_grid * n, true, nullptr},
        {fail, sizeof(int64_t) * n, true, nullptr}};
    const int r = host_windows(*run, arr, [&](const cl_run& w, cudaStream_t st) {
        return window_device(&w, win, n, ns, static_cast<double*>(arr[0].dev), arr[1].dev,
                             static_cast<int8_t*>(arr[2].dev), static_cast<int64_t*>(arr[3].dev),
                             static_cast<int64_t*>(arr[4].dev), n_grid, static_cast<double*>(arr[5].dev),
                             static_cast<int64_t*>(arr[6].dev), st);
    }, prov, "window");
    if (r == 0 && prov)
        std::snprintf(prov->variant, sizeof prov->variant, "indicator window %s H%d K%d",
                      win->kind == CL_WIN_PHASE_ADVANCE ? "phase-advance" : "birkhoff", win->n_windows,
                      win->n_observables);
    return r;
}

}  // extern "C"
