// cl_advance.cu -- `advance_ensemble` (src/Integrators/ensemble.jl:1-45) on the device: `steps` steps of size dt of
// an integrator on the Henon-Heiles flow from every start, one orbit per thread, states only (no tangent).
//
//   SplittingMethod: `advance_n(m, flow, z, dt, steps)` (src/Integrators/stepper.jl:27-48): the kick weight is held
//   back while no drift follows, across the step boundary too, so the last kick of one step and the first of the next
//   are applied as one (a kick-drift-kick leapfrog costs steps + 1 force evaluations).
//   Gauss(3): `advance_checked` once per step (`_run_orbit`, ensemble.jl:5-11): a step whose fixed point fails leaves
//   the all-NaN state (`_nan_state`, gauss.jl:143-147) and ok = false, and the orbit stops there.
//
// States are Julia's Vector{SVector{4, Float64}} (orbit-major, 32 bytes each); ok is Vector{Bool} (one byte each).
// The result of an orbit does not depend on the chunking. Bitwise equal to the oracle's `oracle_advance`.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>

#include "../../include/chaoslab_b200.h"
#include "cl_gauss.cuh"
#include "cl_hostcall.cuh"
#include "cl_split.cuh"

namespace cl {

int capi_fail(int code, const std::string& msg);      // cl_capi.cu
void capi_count_launch();                             // cl_capi.cu

namespace {

struct Table {
    double dt;
    int n;
    double c[CL_MAX_STAGES], d[CL_MAX_STAGES];
};

__global__ void __launch_bounds__(128) advance_split_kernel(const double* __restrict__ x0, double* __restrict__ out,
                                                            uint8_t* __restrict__ ok, int64_t n, int64_t steps,
                                                            const Table m) {
    const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double4 v = reinterpret_cast<const double4*>(x0)[i];
    double z[4] = {v.x, v.y, v.z, v.w};
    double pend = 0.0;
    for (int64_t s = 0; s < steps; ++s) {
#pragma unroll 1
        for (int k = 0; k < m.n; ++k) {
            const double ck = m.c[k];
            if (ck != 0.0) {
                if (pend != 0.0) { SysSplitHH::kick(z, pend * m.dt); pend = 0.0; }
                SysSplitHH::drift(z, ck * m.dt);
            }
            pend = pend + m.d[k];
        }
    }
    if (pend != 0.0) SysSplitHH::kick(z, pend * m.dt);
    reinterpret_cast<double4*>(out)[i] = make_double4(z[0], z[1], z[2], z[3]);
    ok[i] = 1;
}

// advance_n(::CorrectedMethod, n) (stepper.jl:142-152): every step the corrector kick, the base table's step with
// its pending kick flushed at the step's end, the corrector kick
__global__ void __launch_bounds__(128) advance_corrected_kernel(const double* __restrict__ x0,
                                                                double* __restrict__ out, uint8_t* __restrict__ ok,
                                                                int64_t n, int64_t steps, const SysSplitHH m) {
    const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double4 v = reinterpret_cast<const double4*>(x0)[i];
    double z[4] = {v.x, v.y, v.z, v.w};
    for (int64_t s = 0; s < steps; ++s) m.step(z);
    reinterpret_cast<double4*>(out)[i] = make_double4(z[0], z[1], z[2], z[3]);
    ok[i] = 1;
}

__global__ void __launch_bounds__(128) advance_gauss_kernel(const double* __restrict__ x0, double* __restrict__ out,
                                                            uint8_t* __restrict__ ok, int64_t n, int64_t steps,
                                                            const SysGauss3HH g) {
    const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double4 v = reinterpret_cast<const double4*>(x0)[i];
    double z[4] = {v.x, v.y, v.z, v.w};
    uint8_t good = 1;
    for (int64_t s = 0; s < steps; ++s) {
        double inc[4], Y[3][4];
        if (!g.core(z, inc, Y)) {
            const double nan = __longlong_as_double(0x7ff8000000000000LL);
#pragma unroll
            for (int l = 0; l < 4; ++l) z[l] = nan;
            good = 0;
            break;
        }
#pragma unroll
        for (int l = 0; l < 4; ++l) z[l] = z[l] + inc[l];
    }
    reinterpret_cast<double4*>(out)[i] = make_double4(z[0], z[1], z[2], z[3]);
    ok[i] = good;
}

int check_sys(const cl_system* sys) {
    if (!sys) return capi_fail(CL_EINVAL, "sys is NULL");
    if (sys->kind == CL_SYS_HH_SPLIT) {
        if (sys->n_stages < 1 || sys->n_stages > CL_MAX_STAGES)
            return capi_fail(CL_EINVAL, "a table method needs 1 to CL_MAX_STAGES stages");
        for (int k = 0; k < sys->n_stages; ++k)
            if (!std::isfinite(sys->stage_c[k]) || !std::isfinite(sys->stage_d[k]))
                return capi_fail(CL_EINVAL, "the table's weights must be finite");
        if (!(sys->corrector == 0 || (sys->corrector == 1 && std::isfinite(sys->eps))))
            return capi_fail(CL_EINVAL, "corrector must be 0, or 1 with a finite coefficient in eps");
    } else if (sys->kind == CL_SYS_HH_GAUSS) {
        if (sys->gauss_maxiter < 2) return capi_fail(CL_EINVAL, "maxiter must be at least 2");
    } else {
        return capi_fail(CL_EUNSUPPORTED, "advance_ensemble covers IntegratorMap systems (a table method or Gauss(3))");
    }
    if (!std::isfinite(sys->dt)) return capi_fail(CL_EINVAL, "the step size must be finite");
    return 0;
}

}  // namespace
}  // namespace cl

using namespace cl;

extern "C" {

int cl_b200_advance_ensemble_device(const cl_system* sys, int64_t n, const double* x0, double* out, uint8_t* ok,
                                    int64_t steps, void* stream) {
    const int v = check_sys(sys);
    if (v) return v;
    if (n < 0 || steps < 0 || (n > 0 && (!x0 || !out || !ok))) return capi_fail(CL_EINVAL, "bad arguments");
    if ((reinterpret_cast<uintptr_t>(x0) | reinterpret_cast<uintptr_t>(out)) % 32 != 0)
        return capi_fail(CL_EINVAL, "x0 and out must be 32-byte aligned (one SVector{4, Float64} per orbit)");
    if (n == 0) return 0;
    const unsigned blocks = static_cast<unsigned>((n + 127) / 128);
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (sys->kind == CL_SYS_HH_SPLIT && sys->corrector) {
        cl_run r;
        std::memset(&r, 0, sizeof r);
        r.sys = *sys;
        advance_corrected_kernel<<<blocks, 128, 0, st>>>(x0, out, ok, n, steps, SysMaker<SysSplitHH>::make(r, nullptr));
    } else if (sys->kind == CL_SYS_HH_SPLIT) {
        Table m;
        std::memset(&m, 0, sizeof m);
        m.dt = sys->dt;
        m.n = sys->n_stages;
        for (int k = 0; k < m.n; ++k) { m.c[k] = sys->stage_c[k]; m.d[k] = sys->stage_d[k]; }
        advance_split_kernel<<<blocks, 128, 0, st>>>(x0, out, ok, n, steps, m);
    } else {
        SysGauss3HH g;
        g.h = sys->dt;
        g.tol = sys->gauss_tol;
        g.maxiter = sys->gauss_maxiter;
        advance_gauss_kernel<<<blocks, 128, 0, st>>>(x0, out, ok, n, steps, g);
    }
    capi_count_launch();
    const cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? 0 : capi_map_cuda(e, "advance_ensemble launch");
}

int cl_b200_advance_ensemble(const cl_system* sys, int64_t n, const double* x0, double* out, uint8_t* ok,
                             int64_t steps, int64_t chunk, cl_prov* prov) {
    int rc = check_sys(sys);
    if (rc) return rc;
    if (n < 0 || steps < 0 || (n > 0 && (!x0 || !out || !ok))) return capi_fail(CL_EINVAL, "bad arguments");
    const int64_t csz = chunk > 0 ? std::min<int64_t>(chunk, std::max<int64_t>(n, 1)) : std::max<int64_t>(n, 1);
    void *dx = nullptr, *dout = nullptr, *dok = nullptr;
    cudaStream_t st = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    cudaError_t e = cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = pool_alloc(&dx, sizeof(double) * 4 * csz, st);
    if (e == cudaSuccess) e = pool_alloc(&dout, sizeof(double) * 4 * csz, st);
    if (e == cudaSuccess) e = pool_alloc(&dok, csz, st);
    if (e == cudaSuccess) e = cudaEventCreate(&e0);
    if (e == cudaSuccess) e = cudaEventCreate(&e1);
    float total_ms = 0.f;
    int launches = 0;
    for (int64_t lo = 0; lo < n && e == cudaSuccess && rc == 0; lo += csz) {
        const int64_t len = std::min<int64_t>(csz, n - lo);
        cudaMemcpyAsync(dx, x0 + 4 * lo, sizeof(double) * 4 * len, cudaMemcpyHostToDevice, st);
        cudaEventRecord(e0, st);
        rc = cl_b200_advance_ensemble_device(sys, len, static_cast<double*>(dx), static_cast<double*>(dout),
                                             static_cast<uint8_t*>(dok), steps, st);
        cudaEventRecord(e1, st);
        ++launches;
        if (rc) break;
        if (out != x0) touch_pages(out + 4 * lo, sizeof(double) * 4 * len);   // an in-place call keeps its input
        touch_pages(ok + lo, static_cast<size_t>(len));
        cudaMemcpyAsync(out + 4 * lo, dout, sizeof(double) * 4 * len, cudaMemcpyDeviceToHost, st);
        cudaMemcpyAsync(ok + lo, dok, len, cudaMemcpyDeviceToHost, st);
        e = cudaStreamSynchronize(st);
        float ms = 0.f;
        if (e == cudaSuccess) cudaEventElapsedTime(&ms, e0, e1);
        total_ms += ms;
    }
    if (rc == 0 && e != cudaSuccess) rc = capi_map_cuda(e, "advance_ensemble");
    if (rc == 0 && prov) {
        std::memset(prov, 0, sizeof *prov);
        prov->gpu_ms = total_ms;
        prov->launches = launches;
        prov->launch_steps = steps;
        prov->block = 128;
        prov->grid = static_cast<int32_t>((csz + 127) / 128);
        prov->orbits_per_block = 128;
        std::snprintf(prov->variant, sizeof prov->variant, "advance %s",
                      sys->kind == CL_SYS_HH_SPLIT ? "table" : "gauss3");
    }
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    for (void* p : {dx, dout, dok}) pool_free(p, st);
    if (st) cudaStreamDestroy(st);
    return rc;
}

}  // extern "C"
