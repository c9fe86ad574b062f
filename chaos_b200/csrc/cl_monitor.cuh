// cl_monitor.cuh -- the recorders' non-raising monitor, RunMonitor (src/Experiments/run_record.jl:24-43): at each
// handoff the tangent M of the map at the orbit point and the running maxima of |det M - 1|, max|M' Omega M - Omega|
// and max|M|; never fails. Shared by the study recorder and the indicator recorder's kernels.
#pragma once

#include <type_traits>

#include "cl_registry.cuh"

namespace cl {

struct MonState { double det_max, symp_max, M_max; };
static_assert(sizeof(MonState) == 24, "MonState layout");

// The tangent M of the map at x, column-major 2 x 2: standard maps [[1 + K cos x, 1], [K cos x, 1]]
// (standard_map.jl:24-27 as the kernels build it), linear maps A.
template <class Sys>
__device__ __forceinline__ void dense_tangent(const Sys& sys, const double* x, double* M) {
    if constexpr (std::is_same<Sys, SysLinear<2>>::value) {
#pragma unroll
        for (int l = 0; l < 4; ++l) M[l] = sys.A[l];
    } else {
        StdJac J;
        sys.jac(x, J);
        const double o = 1.0;
        M[0] = o + J.c; M[1] = J.c; M[2] = o; M[3] = o;
    }
}

// RunMonitor's step (run_record.jl:37-40): det of a 2 x 2 static matrix M[1] M[4] - M[3] M[2]; M' Omega M by the
// StaticArrays products (the fused chain); Julia's NaN-propagating max.
template <class Sys>
__device__ __forceinline__ void monitor_step(const Sys& sys, const double* x, MonState& m) {
    double M[4];
    dense_tangent(sys, x, M);
    const double edet = fabs((M[0] * M[3] - M[2] * M[1]) - 1.0);
    const double Om[4] = {0.0, -1.0, 1.0, 0.0};
    double P[4], Q[4];
#pragma unroll
    for (int j = 0; j < 2; ++j)
#pragma unroll
        for (int i = 0; i < 2; ++i)   // (M')[i, q] = M[q, i]
            P[i + 2 * j] = fma(M[1 + 2 * i], Om[1 + 2 * j], M[2 * i] * Om[2 * j]);
#pragma unroll
    for (int j = 0; j < 2; ++j)
#pragma unroll
        for (int i = 0; i < 2; ++i) Q[i + 2 * j] = fma(P[i + 2], M[1 + 2 * j], P[i] * M[2 * j]);
    double es = fabs(Q[0] - Om[0]);
#pragma unroll
    for (int l = 1; l < 4; ++l) es = jl_max(es, fabs(Q[l] - Om[l]));
    double mm = fabs(M[0]);
#pragma unroll
    for (int l = 1; l < 4; ++l) mm = jl_max(mm, fabs(M[l]));
    m.det_max = jl_max(m.det_max, edet);
    m.symp_max = jl_max(m.symp_max, es);
    m.M_max = jl_max(m.M_max, mm);
}

}  // namespace cl
