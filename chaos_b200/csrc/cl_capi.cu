// cl_capi.cu -- the C ABI of libchaoslab_b200 (include/chaoslab_b200.h): argument checks with the reference's
// rules, the instance lookup, device buffers, launches and copies, and the error mapping onto FALLBACK_REASONS.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/chaoslab_b200.h"
#include "cl_hostcall.cuh"
#include "cl_registry.cuh"

namespace cl {

namespace {
thread_local std::string g_last_error;
std::atomic<long long> g_launches{0};

std::vector<Instance>& registry_list() {
    static std::vector<Instance> v;
    return v;
}

int fail(int code, const std::string& msg) {
    g_last_error = msg;
    return code;
}

int map_cuda(cudaError_t e, const char* where) {
    std::string m = std::string(where) + ": " + cudaGetErrorString(e);
    switch (e) {
        case cudaErrorMemoryAllocation: return fail(CL_ENOMEM, m);
        case cudaErrorNoDevice: case cudaErrorInsufficientDriver: case cudaErrorInitializationError:
            return fail(CL_ENODEVICE, m);
        case cudaErrorInvalidValue: case cudaErrorInvalidConfiguration: return fail(CL_EINVAL, m);
        case cudaErrorInvalidDeviceFunction: case cudaErrorNoKernelImageForDevice: return fail(CL_EUNSUPPORTED, m);
        default: return fail(CL_EDEVICE_LOST, m);   // launch timeout, illegal address, ... (ChaoslabCUDAExt.jl:36-40)
    }
}

const char* red_token(const cl_reducer& r, char* buf) {
    switch (r.kind) {
        case CL_RED_QR: std::snprintf(buf, 16, "QR%d", r.alg); return buf;
        case CL_RED_BENETTIN: return "BEN";
        case CL_RED_SALI: return "SALI";
        case CL_RED_GALI: return "GALI";
        case CL_RED_MEGNO: std::snprintf(buf, 16, "MEGNO%d", r.replace ? 1 : 0); return buf;
        case CL_RED_FLI: std::snprintf(buf, 16, "FLI%d", r.replace ? 1 : 0); return buf;
        case CL_RED_RLI: std::snprintf(buf, 16, "RLI%d", r.replace ? 1 : 0); return buf;
    }
    return "?";
}

int sys_dim(const cl_system& s, int d) {
    switch (s.kind) {
        case CL_SYS_STANDARD: case CL_SYS_WRAPPED_STANDARD: return 2;
        case CL_SYS_FROESCHLE: case CL_SYS_HH_GAUSS: case CL_SYS_HH_SPLIT: case CL_SYS_WRAPPED_FROESCHLE: return 4;
        case CL_SYS_CHAIN: case CL_SYS_WRAPPED_CHAIN: return 2 * s.n_sites;
        case CL_SYS_LINEAR: return d;
    }
    return -1;
}
// the wrapped maps carry one winding count per coordinate after the coordinates
int sys_state_len(const cl_system& s, int d) {
    const bool wrapped = s.kind == CL_SYS_WRAPPED_STANDARD || s.kind == CL_SYS_WRAPPED_FROESCHLE ||
                         s.kind == CL_SYS_WRAPPED_CHAIN;
    return wrapped ? 2 * sys_dim(s, d) : sys_dim(s, d);
}

int64_t state_bytes_of(const cl_reducer& r, int k) {
    switch (r.kind) {
        case CL_RED_QR: return 16 * k + 72;
        case CL_RED_BENETTIN: return 48;
        case CL_RED_SALI: return 72;
        case CL_RED_GALI: return 24 * k + 32;
        case CL_RED_MEGNO: return 200;
        case CL_RED_FLI: return 96;
        case CL_RED_RLI: return 88;
    }
    return 0;
}

// The checks of `propagate` (src/Tangent/propagate.jl:279-290), `_check_steps` (orbit.jl:66-70) and the reducers'
// `reducer_init` (ArgumentError there), plus the limits of the compiled menu.
int validate(const cl_run& r) {
    char msg[256];
    if (r.abi_version != CL_B200_ABI_VERSION) return fail(CL_EINVAL, "abi_version mismatch");
    if (!(r.tau >= 1 && r.N >= 1 && r.N % r.tau == 0)) {
        std::snprintf(msg, sizeof msg, "N must be a positive multiple of tau, got N = %lld, tau = %d", (long long)r.N, r.tau);
        return fail(CL_EINVAL, msg);
    }
    const int64_t steps = r.steps > 0 ? r.steps : r.N - r.n0;
    if (r.n0 < 0 || r.n0 % r.tau != 0 || steps % r.tau != 0 || r.n0 + steps > r.N || steps <= 0)
        return fail(CL_EINVAL, "launch window must be multiples of tau inside 0..N");
    const int d = sys_dim(r.sys, r.d);
    if (d < 0) return fail(CL_EINVAL, "unknown system kind");
    const bool chain = r.sys.kind == CL_SYS_CHAIN || r.sys.kind == CL_SYS_WRAPPED_CHAIN;
    if (chain && !(r.sys.n_sites >= 2 && r.sys.n_sites <= CL_MAX_DIM / 2))
        return fail(CL_EUNSUPPORTED, "StandardMapChain sites outside the compiled menu (2..8)");
    if (chain && r.sys.ring && r.sys.n_sites < 3) return fail(CL_EINVAL, "a ring needs N >= 3");
    if (r.d != d) {
        std::snprintf(msg, sizeof msg, "d = %d does not match the system dimension %d", r.d, d);
        return fail(CL_EINVAL, msg);
    }
    if (d < 2 || d > CL_MAX_DIM) return fail(CL_EUNSUPPORTED, "dimension outside the compiled menu");
    if (r.s < d) {
        std::snprintf(msg, sizeof msg, "state length %d is below the system dimension %d", r.s, d);
        return fail(CL_EINVAL, msg);
    }
    if (r.s != sys_state_len(r.sys, d)) return fail(CL_EINVAL, "state length does not match the system");
    if (r.sys.kind == CL_SYS_HH_GAUSS) {
        if (r.sys.gauss_maxiter < 2) return fail(CL_EINVAL, "maxiter must be at least 2");
        if (!(std::isfinite(r.sys.dt) && r.sys.dt != 0.0)) return fail(CL_EINVAL, "the step dt must be finite and nonzero");
    }
    if (r.sys.kind == CL_SYS_HH_SPLIT) {
        if (!(r.sys.n_stages >= 1 && r.sys.n_stages <= CL_MAX_STAGES))
            return fail(CL_EUNSUPPORTED, "a splitting table needs 1..CL_MAX_STAGES (128) stages");
        if (!(std::isfinite(r.sys.dt) && r.sys.dt != 0.0)) return fail(CL_EINVAL, "the step dt must be finite and nonzero");
        for (int i = 0; i < r.sys.n_stages; ++i)
            if (!(std::isfinite(r.sys.stage_c[i]) && std::isfinite(r.sys.stage_d[i])))
                return fail(CL_EINVAL, "the splitting table has a non-finite weight");
        if (!(r.sys.corrector == 0 || (r.sys.corrector == 1 && std::isfinite(r.sys.eps))))
            return fail(CL_EINVAL, "corrector must be 0, or 1 with a finite coefficient in eps");
    }
    if (r.n_frames < 1 || r.n_frames > CL_MAX_FRAMES) return fail(CL_EINVAL, "n_frames must be in 1..3");
    if (r.precision != CL_PREC_FP64 && r.precision != CL_PREC_MIXED && r.precision != CL_PREC_MIXED_IND64)
        return fail(CL_EINVAL, "unknown precision");
    for (int f = 0; f < r.n_frames; ++f) {
        const cl_frame& fr = r.frames[f];
        if (!(fr.k >= 1 && fr.k <= d)) {
            std::snprintf(msg, sizeof msg, "k must be in 1:%d, got %d", d, fr.k);
            return fail(CL_EINVAL, msg);
        }
        if (fr.k > CL_MAX_K) return fail(CL_EUNSUPPORTED, "k above the compiled menu (8)");
        if (fr.n_reducers < 0 || fr.n_reducers > CL_MAX_REDUCERS) return fail(CL_EINVAL, "n_reducers must be in 0..4");
        for (int i = 0; i < fr.n_reducers; ++i) {
            const cl_reducer& rd = fr.reducers[i];
            const bool sali_after_gali = rd.kind == CL_RED_SALI && i > 0 && fr.reducers[i - 1].kind == CL_RED_GALI;
            switch (rd.kind) {
                case CL_RED_QR:
                    if (rd.alg < CL_QR_CGS || rd.alg > CL_QR_GIVENS) return fail(CL_EINVAL, "unknown QR algorithm");
                    break;
                case CL_RED_BENETTIN:
                    if (fr.k != 1) return fail(CL_EINVAL, "Benettin needs k = 1");
                    break;
                case CL_RED_SALI:
                    if (fr.k != 2 && !sali_after_gali) return fail(CL_EINVAL, "SALI needs k = 2");
                    break;
                case CL_RED_GALI:
                    if (!(fr.k >= 2 && fr.k <= d)) return fail(CL_EINVAL, "GALI needs 2 <= k <= d");
                    break;
                case CL_RED_MEGNO:
                    if (fr.k != 2) return fail(CL_EINVAL, "MEGNO needs k = 2");
                    break;
                case CL_RED_FLI:
                    if (fr.k != 2) return fail(CL_EINVAL, "FLI needs k = 2");
                    break;
                case CL_RED_RLI:   // reducer_init (rli.jl:45-49); the pair stream doubles d, so it is even
                    if (fr.k != 2) return fail(CL_EINVAL, "RLI needs k = 2");
                    break;
                default: return fail(CL_EINVAL, "unknown reducer kind");
            }
        }
    }
    return 0;
}

int64_t frame_bytes(const cl_frame& f) {
    int64_t b = 0;
    for (int r = 0; r < f.n_reducers; ++r) b += state_bytes_of(f.reducers[r], f.k);
    return b;
}

const Instance* lookup(const cl_run& r) {
    const std::string key = run_key(r);
    const Instance* in = find_instance(key);
    if (!in) fail(CL_EUNSUPPORTED, "no compiled kernel instance for " + key);
    return in;
}

// The per-call device buffers of the host-buffer entry points, from the library's pool on the call's stream,
// returned to it (in stream order) when the call ends.
struct DevBufs {
    cudaStream_t st;
    std::vector<void*> ptrs;
    explicit DevBufs(cudaStream_t s) : st(s) {}
    ~DevBufs() { for (void* p : ptrs) pool_free(p, st); }
    cudaError_t alloc(void** p, size_t bytes) {
        cudaError_t e = pool_alloc(p, bytes, st);
        if (e == cudaSuccess && *p) ptrs.push_back(*p);
        return e;
    }
};

// One stream-ordered memory pool per device, owned by the library: a host-buffer call takes its device buffers
// from it and gives them back when it ends, and the pool keeps the memory (release threshold: never) so the next
// call of the same size allocates nothing from the driver -- a cudaMalloc / cudaFree pair per buffer cost more
// than the copies of the 65536-orbit workload. cl_b200_release_cache returns the kept memory to the driver.
std::mutex g_pool_mu;
constexpr int kMaxDevices = 64;
cudaMemPool_t g_pools[kMaxDevices] = {};
int8_t g_pool_state[kMaxDevices] = {};   // 0 unset, 1 pool, -1 no pool support (plain cudaMalloc)

int device_pool(int dev, cudaMemPool_t* out) {
    *out = nullptr;
    if (dev < 0 || dev >= kMaxDevices) return -1;
    std::lock_guard<std::mutex> g(g_pool_mu);
    if (g_pool_state[dev] == 0) {
        int supported = 0;
        cudaDeviceGetAttribute(&supported, cudaDevAttrMemoryPoolsSupported, dev);
        g_pool_state[dev] = -1;
        if (supported) {
            cudaMemPoolProps props;
            std::memset(&props, 0, sizeof props);
            props.allocType = cudaMemAllocationTypePinned;
            props.handleTypes = cudaMemHandleTypeNone;
            props.location.type = cudaMemLocationTypeDevice;
            props.location.id = dev;
            cudaMemPool_t pool = nullptr;
            if (cudaMemPoolCreate(&pool, &props) == cudaSuccess) {
                uint64_t keep = ~uint64_t(0);
                cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
                g_pools[dev] = pool;
                g_pool_state[dev] = 1;
            } else {
                cudaGetLastError();
            }
        }
    }
    *out = g_pools[dev];
    return g_pool_state[dev];
}

// Memory the device's pool keeps but no call uses: free for the library's next call, so the probe counts it free.
size_t pool_idle_bytes(int dev) {
    std::lock_guard<std::mutex> g(g_pool_mu);
    if (dev < 0 || dev >= kMaxDevices || g_pool_state[dev] != 1) return 0;
    uint64_t reserved = 0, used = 0;
    if (cudaMemPoolGetAttribute(g_pools[dev], cudaMemPoolAttrReservedMemCurrent, &reserved) != cudaSuccess ||
        cudaMemPoolGetAttribute(g_pools[dev], cudaMemPoolAttrUsedMemCurrent, &used) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    return reserved > used ? static_cast<size_t>(reserved - used) : 0;
}

}  // namespace

cudaError_t pool_alloc(void** p, size_t bytes, cudaStream_t st) {
    *p = nullptr;
    if (bytes == 0) return cudaSuccess;
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    cudaMemPool_t pool;
    if (device_pool(dev, &pool) == 1) return cudaMallocFromPoolAsync(p, bytes, pool, st);
    return cudaMalloc(p, bytes);
}

void pool_free(void* p, cudaStream_t st) {
    if (!p) return;
    cudaPointerAttributes at;
    int dev = 0;
    if (cudaPointerGetAttributes(&at, p) == cudaSuccess) dev = at.device;
    cudaMemPool_t pool;
    if (device_pool(dev, &pool) == 1) cudaFreeAsync(p, st);
    else cudaFree(p);
}

void register_instance(const char* key, LaunchFn fn, unsigned mask) { registry_list().push_back(Instance{key, fn, mask}); }

namespace {
std::mutex g_tuned_mu;
std::vector<std::pair<std::string, int>> g_tuned_minb;   // run key + tau -> register budget picked by cl_b200_tune
int tuned_minb(const cl_run& r) {
    const std::string k = run_key(r) + "t" + std::to_string(r.tau);
    std::lock_guard<std::mutex> g(g_tuned_mu);
    for (auto& p : g_tuned_minb) if (p.first == k) return p.second;
    return 0;
}
void set_tuned_minb(const cl_run& r, int m) {
    const std::string k = run_key(r) + "t" + std::to_string(r.tau);
    std::lock_guard<std::mutex> g(g_tuned_mu);
    for (auto& p : g_tuned_minb) if (p.first == k) { p.second = m; return; }
    g_tuned_minb.emplace_back(k, m);
}
}  // namespace

namespace {
// The device's name, cached per device (cudaGetDeviceProperties costs milliseconds; the compute capability and SM
// count come from cudaDeviceGetAttribute).
std::mutex g_name_mu;
std::string g_names[64];
const char* device_name(int dev) {
    std::lock_guard<std::mutex> g(g_name_mu);
    if (dev < 0 || dev >= 64) return "";
    if (g_names[dev].empty()) {
        cudaDeviceProp p;
        g_names[dev] = cudaGetDeviceProperties(&p, dev) == cudaSuccess ? std::string(p.name) : std::string("?");
    }
    return g_names[dev].c_str();
}
}  // namespace

// Shared with the ensemble entry points (cl_ensemble_capi.cu).
const char* capi_device_name(int dev) { return device_name(dev); }
int capi_fail(int code, const std::string& msg) { return fail(code, msg); }
int capi_map_cuda(cudaError_t e, const char* where) { return map_cuda(e, where); }
int capi_validate(const cl_run& r) { return validate(r); }
int64_t capi_frame_bytes(const cl_frame& f) { return frame_bytes(f); }
void capi_count_launch() { g_launches.fetch_add(1); }
const Instance* find_instance(const std::string& key) {
    for (const Instance& in : registry_list())
        if (key == in.key) return &in;
    return nullptr;
}
int instance_count() { return static_cast<int>(registry_list().size()); }
const Instance* instance_at(int i) { return &registry_list()[i]; }

std::string run_key(const cl_run& r) {
    char buf[64];
    std::snprintf(buf, sizeof buf, "s%dd%dp%d|", r.sys.kind, r.d, r.precision);
    std::string k = buf;
    for (int f = 0; f < r.n_frames; ++f) {
        std::snprintf(buf, sizeof buf, "k%d:", r.frames[f].k);
        k += buf;
        for (int i = 0; i < r.frames[f].n_reducers; ++i) {
            char t[16];
            if (i) k += ",";
            k += red_token(r.frames[f].reducers[i], t);
        }
        k += "|";
    }
    return k;
}

// Fill the launch-invariant kernel arguments of a run.
static void base_args(const cl_run& r, int64_t n, KArgs& a) {
    std::memset(&a, 0, sizeof a);
    a.n = n;
    a.N = r.N;
    a.tau = r.tau;
    a.seed = r.seed;
    a.orbit_base = r.orbit_base;
    for (int f = 0; f < r.n_frames; ++f)
        for (int i = 0; i < r.frames[f].n_reducers; ++i) a.prm[f][i].orthogonality_tol = r.frames[f].reducers[i].orthogonality_tol;
}

}  // namespace cl

using namespace cl;

extern "C" {

int cl_b200_check(const cl_run* run) {
    if (!run) return fail(CL_EINVAL, "run is NULL");
    const int v = validate(*run);
    if (v) return v;
    return lookup(*run) ? 0 : CL_EUNSUPPORTED;
}

int64_t cl_b200_state_bytes(const cl_run* run, int32_t frame) {
    if (!run || frame < 0 || frame >= run->n_frames) return 0;
    return frame_bytes(run->frames[frame]);
}

int cl_b200_propagate_device(const cl_run* run, int64_t n_orbits, const cl_buffers* dev, int32_t soa, void* stream) {
    if (!run || !dev) return fail(CL_EINVAL, "NULL argument");
    int v = validate(*run);
    if (v) return v;
    const Instance* in = lookup(*run);
    if (!in) return CL_EUNSUPPORTED;
    if (n_orbits <= 0) return 0;
    KArgs a;
    base_args(*run, n_orbits, a);
    a.n0 = run->n0;
    a.steps = run->steps > 0 ? run->steps : run->N - run->n0;
    a.soa = soa ? 1 : 0;
    a.x_in = run->n0 == 0 ? dev->x0 : dev->x;
    a.x_out = dev->x;
    for (int f = 0; f < run->n_frames; ++f) {
        a.W_in[f] = run->n0 == 0 ? dev->W0[f] : dev->W[f];
        a.W_out[f] = dev->W[f];
        a.states[f] = static_cast<uint64_t*>(dev->states[f]);
        a.code[f] = dev->code[f];
        a.hstep[f] = dev->hstep[f];
        if (!a.x_in || !a.x_out || !a.W_out[f] || !a.code[f] || (frame_bytes(run->frames[f]) > 0 && !a.states[f]))
            return fail(CL_EINVAL, "missing device buffer");
        if (run->n0 > 0 && !a.W_in[f]) return fail(CL_EINVAL, "carried W missing");
    }
    LaunchInfo info{};
    cudaError_t e = in->fn(*run, a, nullptr, static_cast<cudaStream_t>(stream), &info, tuned_minb(*run));
    g_launches.fetch_add(1);
    if (e != cudaSuccess) return map_cuda(e, "orbit kernel launch");
    return 0;
}

constexpr int kMaxVariant = 8;   // variants 1..8 (bit v - 1 of an instance's mask)

// The register budget of a run whose key the tuner has not seen: the compiled variants timed once on a sample of
// the run's own start data (the first min(n, 65536) orbits, 20 handoffs), written into scratch outputs so the inputs
// stay untouched, and the fastest kept for the key. Short runs (where the sample would cost more than ~2 % of the
// run) and single-variant instances keep the first variant.
static int auto_minb(const cl_run& run, const Instance* in, int64_t n, double* dx, double* const* dW0, cudaStream_t st) {
    const int have = tuned_minb(run);
    if (have) return have;
    int variants = 0;
    for (int m = 1; m <= kMaxVariant; ++m) variants += (in->minb_mask >> (m - 1)) & 1u;
    const int64_t ns = std::min<int64_t>(n, 65536);
    const int64_t sample = 20 * static_cast<int64_t>(run.tau);
    const double run_work = static_cast<double>(n) * static_cast<double>(run.N - run.n0);
    const double tune_work = 2.0 * variants * static_cast<double>(ns) * static_cast<double>(sample);
    if (variants < 2 || run.n0 != 0 || tune_work > 0.02 * run_work) return 0;
    for (int f = 0; f < run.n_frames; ++f)
        if (!dW0[f]) return 0;   // seeded frames: the tuner needs explicit start frames
    DevBufs db(st);
    cl_buffers dev;
    std::memset(&dev, 0, sizeof dev);
    dev.x0 = dx;
    if (db.alloc(reinterpret_cast<void**>(&dev.x), sizeof(double) * ns * run.s) != cudaSuccess) return 0;
    for (int f = 0; f < run.n_frames; ++f) {
        const int64_t wb = sizeof(double) * ns * run.d * run.frames[f].k, sb = frame_bytes(run.frames[f]) * ns;
        dev.W0[f] = dW0[f];
        if (db.alloc(reinterpret_cast<void**>(&dev.W[f]), wb) != cudaSuccess ||
            db.alloc(&dev.states[f], static_cast<size_t>(sb)) != cudaSuccess ||
            db.alloc(reinterpret_cast<void**>(&dev.code[f]), ns) != cudaSuccess ||
            db.alloc(reinterpret_cast<void**>(&dev.hstep[f]), sizeof(int64_t) * ns) != cudaSuccess)
            return 0;
    }
    int32_t best = 0;
    if (cl_b200_tune(&run, ns, &dev, 0, sample, st, &best) != 0) return 0;
    return best;
}

int cl_b200_release_cache(void) {
    std::lock_guard<std::mutex> g(g_pool_mu);
    for (int dev = 0; dev < kMaxDevices; ++dev) {
        if (g_pool_state[dev] != 1) continue;
        // every host-buffer call has synchronised its stream before returning, so no buffer is in flight
        const cudaError_t e = cudaMemPoolTrimTo(g_pools[dev], 0);
        if (e != cudaSuccess) return map_cuda(e, "release cache");
    }
    return 0;
}

int cl_b200_propagate(const cl_run* run, int64_t n, const cl_buffers* h, cl_prov* prov) {
    if (!run || !h) return fail(CL_EINVAL, "NULL argument");
    int v = validate(*run);
    if (v) return v;
    const Instance* in = lookup(*run);
    if (!in) return CL_EUNSUPPORTED;
    if (n <= 0) return 0;
    const int nf = run->n_frames;
    const int d = run->d, s = run->s;
    const bool carry = run->n0 > 0;
    if (!h->x || (!carry && !h->x0)) return fail(CL_EINVAL, "missing x buffer");
    cudaStream_t st;
    cudaError_t e = cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking);
    if (e != cudaSuccess) return map_cuda(e, "stream");
    struct StreamGuard { cudaStream_t s; ~StreamGuard() { cudaStreamDestroy(s); } } sg{st};
    DevBufs db(st);
    double* dx = nullptr;
    double* dW[CL_MAX_FRAMES] = {};
    double* dW0[CL_MAX_FRAMES] = {};
    void* dst[CL_MAX_FRAMES] = {};
    int8_t* dcode[CL_MAX_FRAMES] = {};
    int64_t* dhs[CL_MAX_FRAMES] = {};
    if ((e = db.alloc(reinterpret_cast<void**>(&dx), sizeof(double) * n * s)) != cudaSuccess) return map_cuda(e, "alloc");
    for (int f = 0; f < nf; ++f) {
        const int k = run->frames[f].k;
        const int64_t sb = frame_bytes(run->frames[f]);
        if (!h->W[f] || !h->code[f] || (sb > 0 && !h->states[f])) return fail(CL_EINVAL, "missing frame buffer");
        if ((e = db.alloc(reinterpret_cast<void**>(&dW[f]), sizeof(double) * n * d * k)) != cudaSuccess) return map_cuda(e, "alloc");
        if ((e = db.alloc(&dst[f], static_cast<size_t>(sb * n))) != cudaSuccess) return map_cuda(e, "alloc");
        if ((e = db.alloc(reinterpret_cast<void**>(&dcode[f]), n)) != cudaSuccess) return map_cuda(e, "alloc");
        if ((e = db.alloc(reinterpret_cast<void**>(&dhs[f]), sizeof(int64_t) * n)) != cudaSuccess) return map_cuda(e, "alloc");
        if (!carry && h->W0[f]) {
            if ((e = db.alloc(reinterpret_cast<void**>(&dW0[f]), sizeof(double) * n * d * k)) != cudaSuccess) return map_cuda(e, "alloc");
            if ((e = cudaMemcpyAsync(dW0[f], h->W0[f], sizeof(double) * n * d * k, cudaMemcpyHostToDevice, st)) != cudaSuccess) return map_cuda(e, "H2D");
        }
        if (carry) {
            if ((e = cudaMemcpyAsync(dW[f], h->W[f], sizeof(double) * n * d * k, cudaMemcpyHostToDevice, st)) != cudaSuccess) return map_cuda(e, "H2D");
            if (sb && (e = cudaMemcpyAsync(dst[f], h->states[f], sb * n, cudaMemcpyHostToDevice, st)) != cudaSuccess) return map_cuda(e, "H2D");
            if ((e = cudaMemcpyAsync(dcode[f], h->code[f], n, cudaMemcpyHostToDevice, st)) != cudaSuccess) return map_cuda(e, "H2D");
            if (h->hstep[f] && (e = cudaMemcpyAsync(dhs[f], h->hstep[f], sizeof(int64_t) * n, cudaMemcpyHostToDevice, st)) != cudaSuccess) return map_cuda(e, "H2D");
        }
    }
    if ((e = cudaMemcpyAsync(dx, carry ? h->x : h->x0, sizeof(double) * n * s, cudaMemcpyHostToDevice, st)) != cudaSuccess)
        return map_cuda(e, "H2D");

    // Launches of `launch_steps` steps (the reference's step-chunked relaunch, propagate.jl:101-109); the first may
    // start fresh, every later one carries the state in place.
    const int64_t total = run->N - run->n0;
    const int64_t L = run->steps > 0 ? run->steps : total;
    const int minb = auto_minb(*run, in, n, dx, dW0, st);
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaEventRecord(e0, st);
    int64_t launches = 0;
    LaunchInfo info{};
    for (int64_t done = 0; done < total; done += L) {
        cl_run rr = *run;
        rr.n0 = run->n0 + done;
        rr.steps = L < total - done ? L : total - done;
        KArgs a;
        base_args(rr, n, a);
        a.n0 = rr.n0;
        a.steps = rr.steps;
        a.soa = 0;
        a.x_in = dx;
        a.x_out = dx;
        for (int f = 0; f < nf; ++f) {
            a.W_in[f] = rr.n0 == 0 ? dW0[f] : dW[f];
            a.W_out[f] = dW[f];
            a.states[f] = static_cast<uint64_t*>(dst[f]);
            a.code[f] = dcode[f];
            a.hstep[f] = dhs[f];
        }
        e = in->fn(rr, a, nullptr, st, &info, minb);
        g_launches.fetch_add(1);
        ++launches;
        if (e != cudaSuccess) { cudaEventDestroy(e0); cudaEventDestroy(e1); return map_cuda(e, "orbit kernel launch"); }
    }
    cudaEventRecord(e1, st);
    // The inputs are staged (pageable copies return once the source is read), so the outputs' pages can be touched.
    // Only arrays that are outputs alone: an array that was also copied in (a carried launch window, or x given as
    // x0) keeps the caller's values if a kernel or a copy back fails.
    if (!carry) {
        if (h->x != h->x0) touch_pages(h->x, sizeof(double) * n * s);
        for (int f = 0; f < nf; ++f) {
            if (h->W[f] != h->W0[f]) touch_pages(h->W[f], sizeof(double) * n * d * run->frames[f].k);
            touch_pages(h->states[f], static_cast<size_t>(frame_bytes(run->frames[f]) * n));
            touch_pages(h->code[f], static_cast<size_t>(n));
            if (h->hstep[f]) touch_pages(h->hstep[f], sizeof(int64_t) * n);
        }
    }
    if ((e = cudaMemcpyAsync(h->x, dx, sizeof(double) * n * s, cudaMemcpyDeviceToHost, st)) != cudaSuccess) return map_cuda(e, "D2H");
    for (int f = 0; f < nf; ++f) {
        const int k = run->frames[f].k;
        const int64_t sb = frame_bytes(run->frames[f]);
        if ((e = cudaMemcpyAsync(h->W[f], dW[f], sizeof(double) * n * d * k, cudaMemcpyDeviceToHost, st)) != cudaSuccess) return map_cuda(e, "D2H");
        if (sb && (e = cudaMemcpyAsync(h->states[f], dst[f], sb * n, cudaMemcpyDeviceToHost, st)) != cudaSuccess) return map_cuda(e, "D2H");
        if ((e = cudaMemcpyAsync(h->code[f], dcode[f], n, cudaMemcpyDeviceToHost, st)) != cudaSuccess) return map_cuda(e, "D2H");
        if (h->hstep[f] && (e = cudaMemcpyAsync(h->hstep[f], dhs[f], sizeof(int64_t) * n, cudaMemcpyDeviceToHost, st)) != cudaSuccess) return map_cuda(e, "D2H");
    }
    e = cudaStreamSynchronize(st);
    float ms = 0.f;
    if (e == cudaSuccess) cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (e != cudaSuccess) return map_cuda(e, "synchronize");
    if (prov) {
        std::memset(prov, 0, sizeof *prov);
        int dev = 0;
        cudaGetDevice(&dev);
        std::snprintf(prov->device, sizeof prov->device, "%s", device_name(dev));
        std::snprintf(prov->variant, sizeof prov->variant, "%s", in->key);
        prov->launch_steps = L;
        prov->launches = launches;
        prov->gpu_ms = ms;
        prov->block = info.block;
        prov->grid = info.grid;
        prov->regs = info.regs;
        prov->orbits_per_block = info.block;
    }
    return 0;
}

int cl_b200_tune(const cl_run* run, int64_t n_orbits, const cl_buffers* dev, int32_t soa, int64_t sample_steps,
                 void* stream, int32_t* minb_out) {
    if (!run || !dev || n_orbits <= 0) return fail(CL_EINVAL, "bad arguments");
    int v = validate(*run);
    if (v) return v;
    const Instance* in = lookup(*run);
    if (!in) return CL_EUNSUPPORTED;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    cl_run rr = *run;
    const int64_t steps = std::max<int64_t>(rr.tau, (sample_steps > 0 ? sample_steps : 100 * rr.tau) / rr.tau * rr.tau);
    rr.N = steps;
    rr.n0 = 0;
    rr.steps = steps;
    KArgs a;
    base_args(rr, n_orbits, a);
    a.n0 = 0;
    a.steps = steps;
    a.soa = soa ? 1 : 0;
    a.x_in = dev->x0;
    a.x_out = dev->x;
    for (int f = 0; f < rr.n_frames; ++f) {
        a.W_in[f] = dev->W0[f];
        a.W_out[f] = dev->W[f];
        a.states[f] = static_cast<uint64_t*>(dev->states[f]);
        a.code[f] = dev->code[f];
        a.hstep[f] = dev->hstep[f];
        if (!a.x_in || !a.x_out || !a.W_out[f] || !a.code[f] || (frame_bytes(rr.frames[f]) > 0 && !a.states[f]))
            return fail(CL_EINVAL, "missing device buffer");
    }
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    int best = 1;
    float best_ms = 1e30f;
    int rc = 0;
    for (int m = 1; m <= kMaxVariant && rc == 0; ++m) {
        if (!(in->minb_mask & (1u << (m - 1)))) continue;
        float ms = 0.f;
        for (int rep = 0; rep < 2; ++rep) {   // the first run warms up
            cudaEventRecord(e0, st);
            cudaError_t e = in->fn(rr, a, nullptr, st, nullptr, m);
            cudaEventRecord(e1, st);
            if (e != cudaSuccess) { rc = map_cuda(e, "tune launch"); break; }
            cudaEventSynchronize(e1);
            cudaEventElapsedTime(&ms, e0, e1);
        }
        if (rc == 0 && ms < best_ms) { best_ms = ms; best = m; }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (rc) return rc;
    set_tuned_minb(*run, best);
    if (minb_out) *minb_out = best;
    return 0;
}

int32_t cl_b200_variants(const cl_run* run) {
    if (!run || validate(*run) != 0) return 0;
    const Instance* in = find_instance(run_key(*run));
    return in ? static_cast<int32_t>(in->minb_mask) : 0;
}

int cl_b200_set_variant(const cl_run* run, int32_t variant) {
    if (!run) return fail(CL_EINVAL, "run is NULL");
    const int v = validate(*run);
    if (v) return v;
    const Instance* in = lookup(*run);
    if (!in) return CL_EUNSUPPORTED;
    if (variant != 0 && !(variant >= 1 && variant <= kMaxVariant && (in->minb_mask >> (variant - 1)) & 1u))
        return fail(CL_EINVAL, "variant not compiled for this instance");
    set_tuned_minb(*run, variant);
    return 0;
}

int cl_b200_probe(cl_probe* out) {
    if (!out) return fail(CL_EINVAL, "NULL argument");
    std::memset(out, 0, sizeof *out);
    out->loadable = 1;
    int count = 0;
    cudaError_t e = cudaGetDeviceCount(&count);
    if (e != cudaSuccess || count == 0) return fail(CL_ENODEVICE, "no CUDA device");
    int dev = 0;
    cudaGetDevice(&dev);
    int major = 0, minor = 0, smc = 0;
    if ((e = cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, dev)) != cudaSuccess ||
        (e = cudaDeviceGetAttribute(&minor, cudaDevAttrComputeCapabilityMinor, dev)) != cudaSuccess ||
        (e = cudaDeviceGetAttribute(&smc, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess)
        return map_cuda(e, "properties");
    std::snprintf(out->device, sizeof out->device, "%s", device_name(dev));
    out->sm = major * 10 + minor;
    out->sm_count = smc;
    size_t fr = 0, tot = 0;
    if (cudaMemGetInfo(&fr, &tot) == cudaSuccess) { out->free_bytes = fr + pool_idle_bytes(dev); out->total_bytes = tot; }
    out->functional = 1;
    out->compiles = out->sm == 100 ? 1 : 0;   // the cubins are sm_100a only
    return out->compiles ? 0 : fail(CL_EUNSUPPORTED, "device is not sm_100 (B200)");
}

int cl_b200_last_error(char* buf, size_t len) {
    if (buf && len) std::snprintf(buf, len, "%s", g_last_error.c_str());
    return static_cast<int>(g_last_error.size());
}

const char* cl_b200_version(void) { return "libchaoslab_b200 0.1.0 (sm_100a)"; }

int64_t cl_b200_launch_count(void) { return g_launches.load(); }

// Menu introspection for tests: number of compiled instances and the key of instance i.
int32_t cl_b200_menu_size(void) { return instance_count(); }
const char* cl_b200_menu_key(int32_t i) { return (i >= 0 && i < instance_count()) ? instance_at(i)->key : nullptr; }

}  // extern "C"
