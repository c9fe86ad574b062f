// cl_registry.cuh -- the menu of compiled orbit-kernel instances and how one is launched.
//
// Julia specialises `_orbit_kernel!` per (system type, reducer tuple type, element type) at run time; the B200
// library compiles a fixed menu of such specialisations ahead of time (cl_menu_*.cu, generated by gen_menu.py) and
// looks the requested one up by a key built from the cl_run. A run outside the menu is CL_EUNSUPPORTED, which the
// caller maps to the reference's fallback reason 3 ("kernel does not compile for the element type").
#pragma once

#include <cuda_runtime.h>

#include <string>

#include "cl_kernel.cuh"

namespace cl {

struct LaunchInfo { int block, grid, regs; };

typedef cudaError_t (*LaunchFn)(const cl_run& run, const KArgs& a, const double* devA, cudaStream_t st,
                                LaunchInfo* info, int minb);

// An instance and the register budgets it was compiled with (bit b set: blocks-per-SM cap b + 1 available).
struct Instance { const char* key; LaunchFn fn; unsigned minb_mask; };

void register_instance(const char* key, LaunchFn fn, unsigned minb_mask);
const Instance* find_instance(const std::string& key);
int instance_count();
const Instance* instance_at(int i);

// Key of a run: system kind, d, precision, then per frame k and the reducer chain.
std::string run_key(const cl_run& run);

template <class Sys> Sys make_sys(const cl_run& run, const double* devA);
template <> inline SysStandard make_sys<SysStandard>(const cl_run& r, const double*) { SysStandard s; s.K = r.sys.K; return s; }
template <> inline SysWrapped make_sys<SysWrapped>(const cl_run& r, const double*) { SysWrapped s; s.K = r.sys.K; return s; }
template <> inline SysFroeschle make_sys<SysFroeschle>(const cl_run& r, const double*) {
    SysFroeschle s; s.nu = r.sys.nu; s.kappa = r.sys.kappa; s.mu = r.sys.mu; return s;
}
template <> inline SysWrappedFroeschle make_sys<SysWrappedFroeschle>(const cl_run& r, const double*) {
    SysWrappedFroeschle s; s.nu = r.sys.nu; s.kappa = r.sys.kappa; s.mu = r.sys.mu; return s;
}
template <class Sys> struct SysMaker;
template <int DD> struct SysMaker<SysLinear<DD>> {
    static SysLinear<DD> make(const cl_run& r, const double*) {
        SysLinear<DD> s;
        for (int l = 0; l < DD * DD; ++l) s.A[l] = r.sys.A[l];
        return s;
    }
};
template <int NS> struct SysMaker<SysChain<NS>> {
    static SysChain<NS> make(const cl_run& r, const double*) {
        SysChain<NS> s; s.K = r.sys.K; s.eps = r.sys.eps; s.ring = r.sys.ring; return s;
    }
};
template <int NS> struct SysMaker<SysWrappedChain<NS>> {
    static SysWrappedChain<NS> make(const cl_run& r, const double*) {
        SysWrappedChain<NS> s; s.K = r.sys.K; s.eps = r.sys.eps; s.ring = r.sys.ring; return s;
    }
};
template <class Sys> struct SysMaker {
    static Sys make(const cl_run& r, const double* devA) { return make_sys<Sys>(r, devA); }
};

constexpr int ORBIT_BLOCK = 128;

template <class Sys, typename Real, class F0, class F1, class F2, int NF, int MINB>
cudaError_t launch_variant(const cl_run& run, const KArgs& a, const double* devA, cudaStream_t st, LaunchInfo* info) {
    const Sys sys = SysMaker<Sys>::make(run, devA);
    auto k = orbit_kernel<Sys, Real, F0, F1, F2, NF, MINB>;
    const int block = ORBIT_BLOCK;
    const long long grid = (a.n + block - 1) / block;
    k<<<static_cast<unsigned>(grid), block, 0, st>>>(a, sys);
    cudaError_t e = cudaGetLastError();
    if (info) {
        cudaFuncAttributes at;
        if (cudaFuncGetAttributes(&at, k) == cudaSuccess) info->regs = at.numRegs;
        info->block = block;
        info->grid = static_cast<int>(grid);
    }
    return e;
}

// The compiled variants MB... of one instance; an unknown minb runs the first.
template <class Sys, typename Real, class F0, class F1, class F2, int NF, int... MB>
cudaError_t launch_instance(const cl_run& run, const KArgs& a, const double* devA, cudaStream_t st, LaunchInfo* info,
                            int minb) {
    cudaError_t e = cudaErrorInvalidValue;
    bool done = false;
    ((!done && MB == minb ? (e = launch_variant<Sys, Real, F0, F1, F2, NF, MB>(run, a, devA, st, info), done = true)
                          : false), ...);
    if (!done) {
        constexpr int first[] = {MB...};
        return launch_variant<Sys, Real, F0, F1, F2, NF, first[0]>(run, a, devA, st, info);
    }
    return e;
}
template <int... MB> constexpr unsigned minb_mask() { return ((1u << (MB - 1)) | ...); }

struct Registrar {
    Registrar(const char* key, LaunchFn fn, unsigned mask) { register_instance(key, fn, mask); }
};

}  // namespace cl
