// cl_record.cu -- the study recorder on the device (src/Experiments/run_device.jl:43-78, run_record.jl:24-40): the
// variational methods run the shared per-orbit body segment by segment between grid steps, and at every grid step of
// the launch write one row of the record array R[col, g, orbit] (Julia's column-major order, Float64):
//   lambda (k), det_max, symp_max, orth_max, running max of eps_sum, running max of eps_pair, G_max, M_max, state (s)
// from the estimator's finals and the non-raising monitor `RunMonitor` (running maxima of |det M - 1|, the
// symplecticity residual max|M' Omega M - Omega| and max|M|, M the tangent at the handoff point). A failure records
// the grid index whose segment holds it (1-based, 0 = none) and stops the orbit; state, frame, the reducer states
// (estimator, then monitor: Julia's Tuple{state, MonState{Float64}} layout), status and failing step are carried in
// place between launches. Systems: the standard maps (lifted and wrapped) and 2 x 2 linear maps; estimators: Benettin
// (k = 1) and QRSpectrum with CGS, MGS, RGS, Householder or augmented Householder (k = 2).
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

struct RecArgs {
    i64 n, n0, steps, N;
    int tau;
    double* x;            // n x s, in place (x0 at n0 = 0)
    double* W;            // n x 2 k, in place (W0 at n0 = 0)
    uint64_t* states;     // n records: the estimator's state, then MonState
    int8_t* code;
    i64* hstep;
    const i64* grid;      // increasing step counts (multiples of tau)
    int n_grid;
    double* R;            // ncol x n_grid x n, zeroed by the caller before the first launch
    i64* fail;            // n, zeroed by the caller before the first launch
    RedParams prm;
};

// Real = double: the reference's arithmetic; Real = float: the mixed recorder (Float64 orbit, monitor and log sums,
// Float32 frame and QR), as the mixed orbit kernels.
template <class Sys, class Est, int K, typename Real = double>
struct RecOrbit {
    static constexpr int D = Sys::D, S = Sys::S;
    using EstState = typename Est::template State<D, K>;
    double x[S];
    Real W[D * K];
    EstState est;
    MonState mon;

    // _orbit_body (orbit.jl:44-60) over `steps` steps from global step n with the chain (estimator, monitor)
    __device__ __forceinline__ int8_t body(const Sys& sys, i64& n, i64 steps, i64 N, int tau, const RedParams& prm) {
        for (i64 h = 0; h < steps / tau; ++h) {
            for (int t = 0; t < tau; ++t) {
                typename Sys::template JacR<Real> J;
                sys.jac(x, J);
                sys.template apply<K>(J, W);
                sys.forward(x, J);
            }
            n += tau;
            const int8_t c = all_finite_x<D, S>(x) ? (all_finite<D * K>(W) ? STATUS_OK : STATUS_W) : STATUS_STATE;
            if (c != STATUS_OK) return c;
            Est::template step<D, K>(est, n, W, prm);
            monitor_step(sys, x, mon);
            if (Est::template failed<D, K>(est)) return STATUS_REDUCER;
        }
        return n == N ? (all_finite_x<D, S>(x) ? (all_finite<D * K>(W) ? STATUS_OK : STATUS_W) : STATUS_STATE)
                      : STATUS_OK;
    }
};

template <class E> struct EstFinal;
template <> struct EstFinal<RBenettin> {
    static __device__ __forceinline__ void get(const BenettinState& st, double* lam, double& orth, double& gmax) {
        lam[0] = st.n == 0 ? 0.0 : cs_total(st.sum) / static_cast<double>(st.n);
        orth = 0.0;
        gmax = 1.0;
    }
};
template <int ALG> struct EstFinal<RQR<ALG>> {
    static __device__ __forceinline__ void get(const QRState<2>& st, double* lam, double& orth, double& gmax) {
#pragma unroll
        for (int j = 0; j < 2; ++j) lam[j] = st.n == 0 ? 0.0 : cs_total(st.sums[j]) / static_cast<double>(st.n);
        orth = st.orth_max;
        gmax = st.G_max;
    }
};

template <class Sys, class Est, int K, typename Real>
__global__ void __launch_bounds__(128) record_kernel(const RecArgs a, const Sys sys) {
    using O = RecOrbit<Sys, Est, K, Real>;
    constexpr int S = O::S, D = O::D, NCOL = K + 7 + S;
    constexpr int EW = sizeof(typename O::EstState) / 8, MW = sizeof(MonState) / 8;
    const i64 i = static_cast<i64>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= a.n) return;
    if (!(a.n0 == 0 || a.code[i] == STATUS_OK)) return;
    O o;
#pragma unroll
    for (int c = 0; c < S; ++c) o.x[c] = a.x[i * S + c];
#pragma unroll
    for (int l = 0; l < D * K; ++l) o.W[l] = static_cast<Real>(a.W[i * D * K + l]);
    uint64_t* st = a.states + i * (EW + MW);
    uint64_t* ew = reinterpret_cast<uint64_t*>(&o.est);
    uint64_t* mw = reinterpret_cast<uint64_t*>(&o.mon);
#pragma unroll
    for (int w = 0; w < EW; ++w) ew[w] = a.n0 == 0 ? 0ull : st[w];
#pragma unroll
    for (int w = 0; w < MW; ++w) mw[w] = a.n0 == 0 ? 0ull : st[EW + w];
    i64 n = a.n0, h = a.n0;
    int8_t c = STATUS_OK;
    // the grid steps inside the launch: glo = first g with grid[g] > n0, ghi = last g with grid[g] <= n0 + steps
    int glo = 0;
    while (glo < a.n_grid && a.grid[glo] <= a.n0) ++glo;
    int ghi = glo - 1;
    while (ghi + 1 < a.n_grid && a.grid[ghi + 1] <= a.n0 + a.steps) ++ghi;
    double* Ri = a.R + i * static_cast<i64>(NCOL) * a.n_grid;
    for (int g = glo; g <= ghi; ++g) {
        const i64 target = a.grid[g];
        c = o.body(sys, n, target - n, a.N, a.tau, a.prm);
        h = n;
        if (c != STATUS_OK) { a.fail[i] = g + 1; break; }
        // _dev_row! (run_device.jl:10-22)
        double lam[K], orth, gmax;
        EstFinal<Est>::get(o.est, lam, orth, gmax);
        double* row = Ri + static_cast<i64>(g) * NCOL;
#pragma unroll
        for (int j = 0; j < K; ++j) row[j] = lam[j];
        row[K] = o.mon.det_max;
        row[K + 1] = o.mon.symp_max;
        row[K + 2] = orth;
        if constexpr (K == 2) {   // _dev_sumpair!: eps_sum = |l1 + l2|, eps_pair = max_i |l_i + l_(3-i)| = |l1 + l2|
            const double sp = fabs(lam[0] + lam[1]);
            row[K + 3] = g > 0 ? jl_max(row[K + 3 - NCOL], sp) : sp;
            row[K + 4] = g > 0 ? jl_max(row[K + 4 - NCOL], sp) : sp;
        }
        row[K + 5] = gmax;
        row[K + 6] = o.mon.M_max;
#pragma unroll
        for (int j = 0; j < S; ++j) row[K + 7 + j] = o.x[j];
    }
    if (c == STATUS_OK && n < a.n0 + a.steps) {
        c = o.body(sys, n, a.n0 + a.steps - n, a.N, a.tau, a.prm);
        h = n;
        if (c != STATUS_OK) a.fail[i] = ghi + 2;
    }
#pragma unroll
    for (int k2 = 0; k2 < S; ++k2) a.x[i * S + k2] = o.x[k2];
#pragma unroll
    for (int l = 0; l < D * K; ++l) a.W[i * D * K + l] = static_cast<double>(o.W[l]);
#pragma unroll
    for (int w = 0; w < EW; ++w) st[w] = ew[w];
#pragma unroll
    for (int w = 0; w < MW; ++w) st[EW + w] = mw[w];
    a.code[i] = c;
    if (a.hstep) a.hstep[i] = h;
}

typedef cudaError_t (*RecordFn)(const cl_run& run, const RecArgs& a, cudaStream_t st);

template <class Sys, class Est, int K, typename Real>
cudaError_t launch_record(const cl_run& run, const RecArgs& a, cudaStream_t st) {
    const Sys sys = SysMaker<Sys>::make(run, nullptr);
    record_kernel<Sys, Est, K, Real><<<static_cast<unsigned>((a.n + 127) / 128), 128, 0, st>>>(a, sys);
    return cudaGetLastError();
}

template <class Sys, typename Real>
RecordFn record_fn_for(const cl_frame& f) {
    const cl_reducer& r = f.reducers[0];
    if (f.k == 1 && r.kind == CL_RED_BENETTIN) return launch_record<Sys, RBenettin, 1, Real>;
    if (f.k != 2 || r.kind != CL_RED_QR) return nullptr;
    switch (r.alg) {
        case CL_QR_CGS: return launch_record<Sys, RQR<CL_QR_CGS>, 2, Real>;
        case CL_QR_MGS: return launch_record<Sys, RQR<CL_QR_MGS>, 2, Real>;
        case CL_QR_RGS: return launch_record<Sys, RQR<CL_QR_RGS>, 2, Real>;
        case CL_QR_HOUSEHOLDER: return launch_record<Sys, RQR<CL_QR_HOUSEHOLDER>, 2, Real>;
        case CL_QR_AUGMENTED: return launch_record<Sys, RQR<CL_QR_AUGMENTED>, 2, Real>;
    }
    return nullptr;
}

template <typename Real>
RecordFn record_fn_prec(const cl_run& r) {
    switch (r.sys.kind) {
        case CL_SYS_STANDARD: return record_fn_for<SysStandard, Real>(r.frames[0]);
        case CL_SYS_WRAPPED_STANDARD: return record_fn_for<SysWrapped, Real>(r.frames[0]);
        case CL_SYS_LINEAR: return r.d == 2 ? record_fn_for<SysLinear<2>, Real>(r.frames[0]) : nullptr;
    }
    return nullptr;
}

RecordFn record_fn(const cl_run& r) {
    if (r.n_frames != 1 || r.frames[0].n_reducers != 1) return nullptr;
    if (r.precision == CL_PREC_FP64) return record_fn_prec<double>(r);
    if (r.precision == CL_PREC_MIXED) return record_fn_prec<float>(r);
    return nullptr;
}

}  // namespace
}  // namespace cl

using namespace cl;

extern "C" {

int32_t cl_b200_record_columns(const cl_run* run) { return run ? run->frames[0].k + 7 + run->s : -1; }

int64_t cl_b200_record_state_bytes(const cl_run* run) {
    if (!run) return -1;
    const cl_reducer& r = run->frames[0].reducers[0];
    const int64_t est = r.kind == CL_RED_BENETTIN ? 48 : 16 * run->frames[0].k + 72;
    return est + 24;
}

int cl_b200_record_device(const cl_run* run, int64_t n, double* x, double* W, void* states, int8_t* code,
                          int64_t* hstep, const int64_t* grid, int32_t n_grid, double* R, int64_t* fail, void* stream) {
    if (!run || n <= 0 || !x || !W || !states || !code || !grid || n_grid < 1 || !R || !fail)
        return capi_fail(CL_EINVAL, "bad arguments");
    const int v = capi_validate(*run);
    if (v) return v;
    const RecordFn fn = record_fn(*run);
    if (!fn)
        return capi_fail(CL_EUNSUPPORTED, "the recorder covers the standard maps and 2 x 2 linear maps with Benettin "
                                          "(k = 1) or QRSpectrum(CGS, MGS, RGS, Householder, augmented) (k = 2), Float64");
    RecArgs a;
    std::memset(&a, 0, sizeof a);
    a.n = n; a.n0 = run->n0; a.steps = run->steps > 0 ? run->steps : run->N - run->n0; a.N = run->N; a.tau = run->tau;
    a.x = x; a.W = W; a.states = static_cast<uint64_t*>(states); a.code = code; a.hstep = reinterpret_cast<i64*>(hstep);
    a.grid = reinterpret_cast<const i64*>(grid); a.n_grid = n_grid; a.R = R; a.fail = reinterpret_cast<i64*>(fail);
    a.prm.orthogonality_tol = run->frames[0].reducers[0].orthogonality_tol;
    const cudaError_t e = fn(*run, a, static_cast<cudaStream_t>(stream));
    capi_count_launch();
    return e == cudaSuccess ? 0 : capi_map_cuda(e, "record launch");
}

int cl_b200_record(const cl_run* run, int64_t n, double* x, double* W, void* states, int8_t* code, int64_t* hstep,
                   const int64_t* grid, int32_t n_grid, double* R, int64_t* fail, cl_prov* prov) {
    if (!run || n <= 0 || !x || !W || !states || !code || !grid || n_grid < 1 || !R || !fail)
        return capi_fail(CL_EINVAL, "bad arguments");
    const int rc = capi_validate(*run);
    if (rc) return rc;
    if (!record_fn(*run)) return cl_b200_record_device(run, n, x, W, states, code, hstep, grid, n_grid, R, fail, nullptr);
    const int s = run->s, dk = run->d * run->frames[0].k, ncol = cl_b200_record_columns(run);
    std::vector<HostArray> arr = {
        {x, sizeof(double) * s * n, true, nullptr},
        {W, sizeof(double) * dk * n, true, nullptr},
        {states, static_cast<size_t>(cl_b200_record_state_bytes(run) * n), true, nullptr},
        {code, static_cast<size_t>(n), true, nullptr},
        {hstep, sizeof(int64_t) * n, true, nullptr},
        {const_cast<int64_t*>(grid), sizeof(int64_t) * n_grid, false, nullptr},
        {R, sizeof(double) * ncol * n_grid * n, true, nullptr},
        {fail, sizeof(int64_t) * n, true, nullptr}};
    const int r = host_windows(*run, arr, [&](const cl_run& w, cudaStream_t st) {
        return cl_b200_record_device(&w, n, static_cast<double*>(arr[0].dev), static_cast<double*>(arr[1].dev),
                                     arr[2].dev, static_cast<int8_t*>(arr[3].dev), static_cast<int64_t*>(arr[4].dev),
                                     static_cast<int64_t*>(arr[5].dev), n_grid, static_cast<double*>(arr[6].dev),
                                     static_cast<int64_t*>(arr[7].dev), st);
    }, prov, "record");
    if (r == 0 && prov) std::snprintf(prov->variant, sizeof prov->variant, "record k%d s%d", run->frames[0].k, s);
    return r;
}

}  // extern "C"
