// cl_indicator.cu -- the indicator recorder's series kernel on the device (src/Experiments/run_indicator_device.jl:
// 13-60, run_indicator_record.jl:39-75) for the tangent kind: a chain of indicator members (SALI, FLI, MEGNO; every
// member but the last non-replacing, the last replacing, E23) followed by the non-raising monitor, run segment by
// segment between the grid steps on a k = 2 frame; at every grid step one row of R[col, g, orbit] (Float64):
//   the members' columns (E24: SALI sali, L; FLI fli, fli1; MEGNO Y_1, Ybar_1, Ybar20_1, Y_2, Ybar_2, Ybar20_2),
//   det_max, symp_max, M_max of the monitor, then the first ns coordinates of the orbit point.
// A failure stores the 1-based grid index whose segment holds it and stops the orbit; everything is carried in place.
// The pair kind runs the same body on PairMap(sys) (src/Systems/pair.jl:9-68) with the members RLI and MEGNO on the
// block frame, the monitor reading orbit A (run_indicator_record.jl:6-10).
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <string>
#include <type_traits>
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
int64_t capi_frame_bytes(const cl_frame& f);          // cl_capi.cu
std::string run_key(const cl_run& r);                 // cl_capi.cu

namespace {

struct IndArgs {
    i64 n, n0, steps, N;
    int tau, ns;
    double* x;
    double* W;
    uint64_t* states;     // the members' states, then MonState
    int8_t* code;
    i64* hstep;
    const i64* grid;
    int n_grid, ncol;
    double* R;
    i64* fail;
    RedParams prm[CL_MAX_REDUCERS];
};

// _put! (run_indicator_record.jl:40-56): a member's columns from its reducer_final
template <class R> struct Put;
template <> struct Put<RSALI> {
    static constexpr int cols = 2;
    static __device__ __forceinline__ void put(const SALIState& st, double* row) {   // sali.jl:55-59
        row[0] = st.sali;
        row[1] = st.n == 0 ? 0.0 : -((st.s1.s + st.s2.s) + (st.s1.c + st.s2.c));
    }
};
template <bool REP> struct Put<RFLI<REP>> {
    static constexpr int cols = 2;
    static __device__ __forceinline__ void put(const FLIState& st, double* row) { row[0] = st.fB; row[1] = st.f1; }
};
template <bool REP> struct Put<RMEGNO<REP>> {
    static constexpr int cols = 6;
    // megno.jl:97-102: Y = 2 R1 / n, Ybar = Q / K, Ybar20 = tau Q2 / n^3 with tau = n / K (0 when K = 0)
    static __device__ __forceinline__ void series(const MegnoSums& m, i64 n, i64 K, double* out) {
        if (K == 0) { out[0] = out[1] = out[2] = 0.0; return; }
        const double tn = static_cast<double>(n);
        out[0] = 2 * cs_total(m.R1) / tn;
        out[1] = cs_total(m.Q) / static_cast<double>(K);
        out[2] = static_cast<double>(n / K) * cs_total(m.Q2) / (tn * tn * tn);
    }
    static __device__ __forceinline__ void put(const MEGNOState& st, double* row) {
        series(st.c1, st.n, st.K, row);
        series(st.c2, st.n, st.K, row + 3);
    }
};

template <bool REP> struct Put<RRLI<REP>> {
    static constexpr int cols = 2;
    // reducer_final (rli.jl:98-101): DL at the last handoff and RLI = Q / K, zeros before the first handoff
    static __device__ __forceinline__ void put(const RLIState& st, double* row) {
        row[0] = st.K == 0 ? 0.0 : fabs((st.sB.s - st.sA.s) + (st.sB.c - st.sA.c)) / static_cast<double>(st.n);
        row[1] = st.K == 0 ? 0.0 : cs_total(st.Q) / static_cast<double>(st.K);
    }
};

// PairMap(sys) (pair.jl:9-68): the state (A; B), each half advanced by the base map alone; the tangent acts block by
// block (PairTangent * W, pair.jl:37-41), the rows of each block multiplied by the base's own product, the zero
// blocks never touched.
template <class Base>
struct SysPair {
    static constexpr int Db = Base::D, Sb = Base::S, D = 2 * Db, S = 2 * Sb;
    struct Jac { typename Base::Jac A, B; };
    Base base;
    __device__ __forceinline__ void jac(const double* x, Jac& J) const {
        base.jac(x, J.A);
        base.jac(x + Sb, J.B);
    }
    template <int KK>
    __device__ __forceinline__ void apply(const Jac& J, double* W) const {
        double Wa[Db * KK], Wb[Db * KK];
#pragma unroll
        for (int j = 0; j < KK; ++j)
#pragma unroll
            for (int l = 0; l < Db; ++l) { Wa[l + Db * j] = W[l + D * j]; Wb[l + Db * j] = W[Db + l + D * j]; }
        base.template apply<KK>(J.A, Wa);
        base.template apply<KK>(J.B, Wb);
#pragma unroll
        for (int j = 0; j < KK; ++j)
#pragma unroll
            for (int l = 0; l < Db; ++l) { W[l + D * j] = Wa[l + Db * j]; W[Db + l + D * j] = Wb[l + Db * j]; }
    }
    __device__ __forceinline__ void forward(double* x, const Jac& J) const {
        base.forward(x, J.A);
        base.forward(x + Sb, J.B);
    }
};

// The map whose tangent the monitor reads at the orbit point: the system itself, or the base map at orbit A.
template <class Sys> __device__ __forceinline__ const Sys& monitored(const Sys& s) { return s; }
template <class Base> __device__ __forceinline__ const Base& monitored(const SysPair<Base>& s) { return s.base; }

// _put_members! over the compile-time chain
template <int D, int K>
__device__ __forceinline__ int put_members(const Chain<D, K>&, double*) { return 0; }
template <int D, int K, class R, class... Rs>
__device__ __forceinline__ int put_members(const Chain<D, K, R, Rs...>& ch, double* row) {
    Put<R>::put(ch.head, row);
    return Put<R>::cols + put_members(ch.tail, row + Put<R>::cols);
}

// One orbit: point, frame, member states, monitor; the orbit body over a segment (orbit.jl:44-60) with the chain
// (members..., monitor)
template <class Sys, class F>
struct IndOrbit {
    static constexpr int D = Sys::D, S = Sys::S, K = F::K;
    using Ch = typename F::template Chain_<D>;
    double x[S], W[D * K];
    Ch ch;
    MonState mon;
    __device__ __forceinline__ int8_t body(const Sys& sys, i64& n, i64 steps, const IndArgs& a) {
        for (i64 hh = 0; hh < steps / a.tau; ++hh) {
            for (int t = 0; t < a.tau; ++t) {
                typename Sys::Jac J;
                sys.jac(x, J);
                sys.template apply<K>(J, W);
                sys.forward(x, J);
            }
            n += a.tau;
            const int8_t cc = all_finite_x<D, S>(x) ? (all_finite<D * K>(W) ? STATUS_OK : STATUS_W) : STATUS_STATE;
            if (cc != STATUS_OK) return cc;
            ch.step(n, W, a.prm);
            monitor_step(monitored(sys), x, mon);
            if (ch.failed()) return STATUS_REDUCER;
        }
        return n == a.N ? (all_finite_x<D, S>(x) ? (all_finite<D * K>(W) ? STATUS_OK : STATUS_W) : STATUS_STATE)
                        : STATUS_OK;
    }
};

template <class Sys, class F>
__global__ void __launch_bounds__(128) ind_series_kernel(const IndArgs a, const Sys sys) {
    using O = IndOrbit<Sys, F>;
    constexpr int D = O::D, S = O::S, K = O::K;
    constexpr int CW = O::Ch::bytes / 8, MW = sizeof(MonState) / 8;
    const i64 i = static_cast<i64>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= a.n) return;
    if (!(a.n0 == 0 || a.code[i] == STATUS_OK)) return;
    O o;
#pragma unroll
    for (int c = 0; c < S; ++c) o.x[c] = a.x[i * S + c];
#pragma unroll
    for (int l = 0; l < D * K; ++l) o.W[l] = a.W[i * D * K + l];
    uint64_t* st = a.states + i * (CW + MW);
    uint64_t* mw = reinterpret_cast<uint64_t*>(&o.mon);
    if (a.n0 == 0) {
        o.ch.zero();
#pragma unroll
        for (int w = 0; w < MW; ++w) mw[w] = 0ull;
    } else {
        o.ch.load(st);
#pragma unroll
        for (int w = 0; w < MW; ++w) mw[w] = st[CW + w];
    }
    i64 n = a.n0, h = a.n0;
    int8_t c = STATUS_OK;
    int glo = 0;
    while (glo < a.n_grid && a.grid[glo] <= a.n0) ++glo;
    int ghi = glo - 1;
    while (ghi + 1 < a.n_grid && a.grid[ghi + 1] <= a.n0 + a.steps) ++ghi;
    double* Ri = a.R + i * static_cast<i64>(a.ncol) * a.n_grid;
    for (int g = glo; g <= ghi; ++g) {
        c = o.body(sys, n, a.grid[g] - n, a);
        h = n;
        if (c != STATUS_OK) { a.fail[i] = g + 1; break; }
        double* row = Ri + static_cast<i64>(g) * a.ncol;
        const int off = put_members(o.ch, row);
        row[off] = o.mon.det_max;
        row[off + 1] = o.mon.symp_max;
        row[off + 2] = o.mon.M_max;
#pragma unroll
        for (int j = 0; j < S; ++j)
            if (j < a.ns) row[off + 3 + j] = o.x[j];
    }
    if (c == STATUS_OK && n < a.n0 + a.steps) {
        c = o.body(sys, n, a.n0 + a.steps - n, a);
        h = n;
        if (c != STATUS_OK) a.fail[i] = ghi + 2;
    }
#pragma unroll
    for (int k2 = 0; k2 < S; ++k2) a.x[i * S + k2] = o.x[k2];
#pragma unroll
    for (int l = 0; l < D * K; ++l) a.W[i * D * K + l] = o.W[l];
    o.ch.store(st);
#pragma unroll
    for (int w = 0; w < MW; ++w) st[CW + w] = mw[w];
    a.code[i] = c;
    if (a.hstep) a.hstep[i] = h;
}

typedef cudaError_t (*IndFn)(const cl_run& run, const IndArgs& a, cudaStream_t st);

template <class Sys> struct IndMaker {
    static Sys make(const cl_run& run) { return SysMaker<Sys>::make(run, nullptr); }
};
template <class Base> struct IndMaker<SysPair<Base>> {
    static SysPair<Base> make(const cl_run& run) {
        SysPair<Base> s;
        s.base = SysMaker<Base>::make(run, nullptr);
        return s;
    }
};

template <class Sys, class F>
cudaError_t launch_ind(const cl_run& run, const IndArgs& a, cudaStream_t st) {
    const Sys sys = IndMaker<Sys>::make(run);
    ind_series_kernel<Sys, F><<<static_cast<unsigned>((a.n + 127) / 128), 128, 0, st>>>(a, sys);
    return cudaGetLastError();
}

struct IndEntry { const char* chain; IndFn std, wrapped, linear; int cols; };

template <class F, int COLS>
constexpr IndEntry entry(const char* chain) {
    return IndEntry{chain, launch_ind<SysStandard, F>, launch_ind<SysWrapped, F>, launch_ind<SysLinear<2>, F>, COLS};
}

// The member chains of the compiled menu (the last member replacing; SALI has one form): the seven tangent chains
// the reference's recorder specs name (test/experiments/ex_d86_chains.jl:4), then the other orders of two members
// and MEGNO, FLI, SALI.
const IndEntry kChains[] = {
    entry<Frame<2, RSALI>, 2>("SALI"),
    entry<Frame<2, RFLI<false>, RSALI>, 4>("FLI0,SALI"),
    entry<Frame<2, RMEGNO<false>, RSALI>, 8>("MEGNO0,SALI"),
    entry<Frame<2, RFLI<false>, RMEGNO<false>, RSALI>, 10>("FLI0,MEGNO0,SALI"),
    entry<Frame<2, RFLI<true>>, 2>("FLI1"),
    entry<Frame<2, RMEGNO<true>>, 6>("MEGNO1"),
    entry<Frame<2, RFLI<false>, RMEGNO<true>>, 8>("FLI0,MEGNO1"),
    entry<Frame<2, RMEGNO<false>, RFLI<false>, RSALI>, 10>("MEGNO0,FLI0,SALI"),
    entry<Frame<2, RMEGNO<false>, RFLI<true>>, 8>("MEGNO0,FLI1"),
    entry<Frame<2, RSALI, RMEGNO<true>>, 8>("SALI,MEGNO1"),
    entry<Frame<2, RSALI, RFLI<true>>, 4>("SALI,FLI1"),
};

template <class F, int COLS>
constexpr IndEntry pair_entry(const char* chain) {
    return IndEntry{chain, launch_ind<SysPair<SysStandard>, F>, launch_ind<SysPair<SysWrapped>, F>,
                    launch_ind<SysPair<SysLinear<2>>, F>, COLS};
}

// The pair chains of the reference's recorder specs (test/experiments/ex_d86_chains.jl:5).
const IndEntry kPairChains[] = {
    pair_entry<Frame<2, RRLI<true>>, 2>("RLI1"),
    pair_entry<Frame<2, RRLI<false>, RMEGNO<true>>, 8>("RLI0,MEGNO1"),
    pair_entry<Frame<2, RMEGNO<false>, RRLI<true>>, 8>("MEGNO0,RLI1"),
};

// "k2:MEGNO0,SALI|" of the run's key -> the member chain
const IndEntry* find_chain(const cl_run& r, bool pair) {
    const std::string key = run_key(r);
    const size_t a = key.find("|k2:");
    if (a == std::string::npos) return nullptr;
    const size_t b = key.find('|', a + 1);
    const std::string chain = key.substr(a + 4, b - a - 4);
    if (pair) {
        for (const IndEntry& e : kPairChains)
            if (chain == e.chain) return &e;
    } else {
        for (const IndEntry& e : kChains)
            if (chain == e.chain) return &e;
    }
    return nullptr;
}

}  // namespace
}  // namespace cl

using namespace cl;

extern "C" {

int32_t cl_b200_indicator_columns(const cl_run* run, int32_t ns) {
    if (!run) return -1;
    const IndEntry* e = find_chain(*run, false);
    return e ? e->cols + 3 + ns : -1;
}

int32_t cl_b200_indicator_pair_columns(const cl_run* run, int32_t ns) {
    if (!run) return -1;
    const IndEntry* e = find_chain(*run, true);
    return e ? e->cols + 3 + ns : -1;
}

int64_t cl_b200_indicator_state_bytes(const cl_run* run) {
    if (!run || run->n_frames < 1) return -1;
    return capi_frame_bytes(run->frames[0]) + static_cast<int64_t>(sizeof(MonState));
}

}  // extern "C"

namespace {
int indicator_device(const cl_run* run, bool pair, int64_t n, int32_t ns, double* x, double* W, void* states,
                     int8_t* code, int64_t* hstep, const int64_t* grid, int32_t n_grid, double* R, int64_t* fail,
                     void* stream) {
    if (!run || n <= 0 || !x || !W || !states || !code || !grid || n_grid < 1 || !R || !fail || ns < 0)
        return capi_fail(CL_EINVAL, "bad arguments");
    const int v = capi_validate(*run);
    if (v) return v;
    if (ns > (pair ? 2 : 1) * run->s) return capi_fail(CL_EINVAL, "ns exceeds the state length");
    const IndEntry* e = find_chain(*run, pair);
    if (!e || run->n_frames != 1 || run->frames[0].k != 2 || run->precision != CL_PREC_FP64)
        return capi_fail(CL_EUNSUPPORTED, "indicator chain outside the compiled menu");
    IndFn fn = run->sys.kind == CL_SYS_STANDARD ? e->std : run->sys.kind == CL_SYS_WRAPPED_STANDARD ? e->wrapped
             : (run->sys.kind == CL_SYS_LINEAR && run->d == 2) ? e->linear : nullptr;
    if (!fn) return capi_fail(CL_EUNSUPPORTED, "the indicator recorder covers the standard maps and 2 x 2 linear maps");
    IndArgs a;
    std::memset(&a, 0, sizeof a);
    a.n = n; a.n0 = run->n0; a.steps = run->steps > 0 ? run->steps : run->N - run->n0; a.N = run->N; a.tau = run->tau;
    a.ns = ns; a.x = x; a.W = W; a.states = static_cast<uint64_t*>(states); a.code = code;
    a.hstep = reinterpret_cast<i64*>(hstep); a.grid = reinterpret_cast<const i64*>(grid); a.n_grid = n_grid;
    a.ncol = e->cols + 3 + ns; a.R = R; a.fail = reinterpret_cast<i64*>(fail);
    for (int r = 0; r < run->frames[0].n_reducers; ++r) a.prm[r].orthogonality_tol = run->frames[0].reducers[r].orthogonality_tol;
    const cudaError_t err = fn(*run, a, static_cast<cudaStream_t>(stream));
    capi_count_launch();
    return err == cudaSuccess ? 0 : capi_map_cuda(err, "indicator launch");
}

int indicator_host(const cl_run* run, bool pair, int64_t n, int32_t ns, double* x, double* W, void* states,
                   int8_t* code, int64_t* hstep, const int64_t* grid, int32_t n_grid, double* R, int64_t* fail,
                   cl_prov* prov) {
    if (!run || n <= 0 || !x || !W || !states || !code || !grid || n_grid < 1 || !R || !fail || ns < 0)
        return capi_fail(CL_EINVAL, "bad arguments");
    int rc = capi_validate(*run);
    if (rc) return rc;
    const int ncol = pair ? cl_b200_indicator_pair_columns(run, ns) : cl_b200_indicator_columns(run, ns);
    const int mult = pair ? 2 : 1;
    if (ncol < 0 || ns > mult * run->s)
        return indicator_device(run, pair, n, ns, x, W, states, code, hstep, grid, n_grid, R, fail, nullptr);
    const int s = mult * run->s, dk = mult * run->d * run->frames[0].k;
    std::vector<HostArray> arr = {
        {x, sizeof(double) * s * n, true, nullptr},
        {W, sizeof(double) * dk * n, true, nullptr},
        {states, static_cast<size_t>(cl_b200_indicator_state_bytes(run) * n), true, nullptr},
        {code, static_cast<size_t>(n), true, nullptr},
        {hstep, sizeof(int64_t) * n, true, nullptr},
        {const_cast<int64_t*>(grid), sizeof(int64_t) * n_grid, false, nullptr},
        {R, sizeof(double) * ncol * n_grid * n, true, nullptr},
        {fail, sizeof(int64_t) * n, true, nullptr}};
    const int r = host_windows(*run, arr, [&](const cl_run& w, cudaStream_t st) {
        return indicator_device(&w, pair, n, ns, static_cast<double*>(arr[0].dev), static_cast<double*>(arr[1].dev),
                                arr[2].dev, static_cast<int8_t*>(arr[3].dev), static_cast<int64_t*>(arr[4].dev),
                                static_cast<int64_t*>(arr[5].dev), n_grid, static_cast<double*>(arr[6].dev),
                                static_cast<int64_t*>(arr[7].dev), st);
    }, prov, "indicator");
    if (r == 0 && prov)
        std::snprintf(prov->variant, sizeof prov->variant, "indicator%s %d cols s%d", pair ? " pair" : "", ncol, s);
    return r;
}

}  // namespace

extern "C" {

int cl_b200_indicator_device(const cl_run* run, int64_t n, int32_t ns, double* x, double* W, void* states,
                             int8_t* code, int64_t* hstep, const int64_t* grid, int32_t n_grid, double* R,
                             int64_t* fail, void* stream) {
    return indicator_device(run, false, n, ns, x, W, states, code, hstep, grid, n_grid, R, fail, stream);
}

int cl_b200_indicator(const cl_run* run, int64_t n, int32_t ns, double* x, double* W, void* states, int8_t* code,
                      int64_t* hstep, const int64_t* grid, int32_t n_grid, double* R, int64_t* fail, cl_prov* prov) {
    return indicator_host(run, false, n, ns, x, W, states, code, hstep, grid, n_grid, R, fail, prov);
}

int cl_b200_indicator_pair_device(const cl_run* run, int64_t n, int32_t ns, double* z, double* W, void* states,
                                  int8_t* code, int64_t* hstep, const int64_t* grid, int32_t n_grid, double* R,
                                  int64_t* fail, void* stream) {
    return indicator_device(run, true, n, ns, z, W, states, code, hstep, grid, n_grid, R, fail, stream);
}

int cl_b200_indicator_pair(const cl_run* run, int64_t n, int32_t ns, double* z, double* W, void* states,
                           int8_t* code, int64_t* hstep, const int64_t* grid, int32_t n_grid, double* R,
                           int64_t* fail, cl_prov* prov) {
    return indicator_host(run, true, n, ns, z, W, states, code, hstep, grid, n_grid, R, fail, prov);
}

}  // extern "C"
