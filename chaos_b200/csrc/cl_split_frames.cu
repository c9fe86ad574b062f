// cl_split_frames.cu -- the split-precision orbit kernel for the coupled-maps ensemble (cl_split_frames.cuh): the
// FroeschleMap orbit with a QRSpectrum(HouseholderQR) frame in Float32 and a GALI_4 + SALI frame in Float64, under
// the run key of precision CL_PREC_MIXED_IND64. The launch window, relaunch carry, frozen failed orbits, status codes and
// the records' layouts are those of the plain kernel (cl_kernel.cuh, after src/Tangent/propagate.jl:32-50).
#include <cuda_runtime.h>

#include "cl_registry.cuh"
#include "cl_split_frames.cuh"

namespace cl {
namespace {

using split::GSSlot;
using split::QRSlot;

constexpr int D = 4, K = 4;
constexpr int QWORDS = static_cast<int>(sizeof(QRState<4>) / 8);            // 17
constexpr int GWORDS = static_cast<int>(sizeof(GALIFrameState<4, true>) / 8);   // 25
// per-thread slot: the reducer fields, then room to park the point and the Float32 frame while the Float64 frame's
// handoff runs (its Gram-Schmidt needs the registers); an odd number of 8-byte words, so the 16 threads of a
// half-warp hit distinct bank pairs
constexpr int PARK_BYTES = 4 * 8 + 16 * 4;
constexpr int SLOT_BYTES = ((static_cast<int>(sizeof(QRSlot) + sizeof(GSSlot)) + PARK_BYTES) / 8 | 1) * 8;
static_assert(sizeof(QRSlot) % 8 == 0 && sizeof(GSSlot) % 8 == 0, "slot layout");

template <typename T>
__device__ __forceinline__ void load_frame(const KArgs& a, int f, i64 i, bool fresh, T* W) {
    const i64 so = a.soa ? 1 : D * K, sc = a.soa ? a.n : 1;
    if (fresh && !a.W_in[f]) {
        seeded_frame<D, K>(a.seed, a.orbit_base + i + 1, W);
        return;
    }
#pragma unroll
    for (int l = 0; l < D * K; ++l) W[l] = static_cast<T>(a.W_in[f][i * so + l * sc]);
}
template <typename T>
__device__ __forceinline__ void store_frame(const KArgs& a, int f, i64 i, const T* W) {
    const i64 so = a.soa ? 1 : D * K, sc = a.soa ? a.n : 1;
#pragma unroll
    for (int l = 0; l < D * K; ++l) a.W_out[f][i * so + l * sc] = static_cast<double>(W[l]);
}
// the Float64 frame as store_frame left it in the output (the unit columns of its last successful handoff)
__device__ __forceinline__ void load_stored64(const KArgs& a, int f, i64 i, double* W) {
    const i64 so = a.soa ? 1 : D * K, sc = a.soa ? a.n : 1;
#pragma unroll
    for (int l = 0; l < D * K; ++l) W[l] = a.W_out[f][i * so + l * sc];
}

// the Float32 frame holds no non-finite entry (a NaN or infinity turns the fma chain's zero into NaN)
__device__ __forceinline__ bool finite32(const float* W) {
    float z = 0.0f;
#pragma unroll
    for (int l = 0; l < D * K; ++l) z = __fmaf_rn(W[l], 0.0f, z);
    return z == 0.0f;
}
// the Float64 frame holds no non-finite entry: the largest exponent field is below the all-ones one
__device__ __forceinline__ bool finite64(const double* W) {
    unsigned m = 0;
#pragma unroll
    for (int l = 0; l < D * K; ++l) m = max(m, static_cast<unsigned>(__double2hiint(W[l])) & 0x7ff00000u);
    return m != 0x7ff00000u;
}
__device__ __forceinline__ bool finite_x(const double* x) {
    return isfin(x[0]) && isfin(x[1]) && isfin(x[2]) && isfin(x[3]);
}

// Blocks of 64 threads: 65536 orbits are 1024 blocks, one wave of 148 SMs at 7 blocks per SM. Registers are
// allocated per scheduler (16384 each), so 128 registers a thread hold 4 warps per scheduler, the 3.5 warps of that
// ensemble; REGS is the budget of the variant.
constexpr int SPLIT_BLOCK = 64;

template <int REGS>
__global__ void __maxnreg__(REGS) split_frames_kernel(const KArgs a, const SysFroeschle sys) {
    extern __shared__ __align__(16) unsigned char slots[];
    QRSlot& q = *reinterpret_cast<QRSlot*>(slots + threadIdx.x * SLOT_BYTES);
    GSSlot& g = *reinterpret_cast<GSSlot*>(slots + threadIdx.x * SLOT_BYTES + sizeof(QRSlot));
    double* park_x = reinterpret_cast<double*>(slots + threadIdx.x * SLOT_BYTES + sizeof(QRSlot) + sizeof(GSSlot));
    float* park_w = reinterpret_cast<float*>(park_x + 4);
    const i64 i = static_cast<i64>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= a.n) return;
    const bool fresh = a.n0 == 0;
    const i64 xso = a.soa ? 1 : 4, xsc = a.soa ? a.n : 1;
    double x[4];
#pragma unroll
    for (int c = 0; c < 4; ++c) x[c] = a.x_in[i * xso + c * xsc];

    // frame 0: QRSpectrum(HouseholderQR), Float32; frame 1: GALI + SALI, Float64
    float W0[16];
    double W1[16];
    load_frame(a, 0, i, fresh, W0);
    load_frame(a, 1, i, fresh, W1);
    int8_t code0 = STATUS_OK, code1 = STATUS_OK;
    i64 hstep0 = 0, hstep1 = 0;
    const QRState<4>* gq = reinterpret_cast<const QRState<4>*>(a.states[0] + i * QWORDS);
    const GALIFrameState<4, true>* gg = reinterpret_cast<const GALIFrameState<4, true>*>(a.states[1] + i * GWORDS);
    if (fresh) {
        q.G_max = 0.0; q.orth_max = 0.0; q.value = 0.0; q.threshold = 0.0;
        q.n = 0; q.count_max = 0; q.column = 0; q.step = 0; q.code = 0;
        g.gali[0] = g.gali[1] = g.gali[2] = 0.0; g.gvalue = 0.0; g.svalue = 0.0; g.sali = 0.0;
        g.gn = 0; g.gstep = 0; g.gcolumn = 0; g.sn = 0; g.sstep = 0; g.gcode = 0; g.scode = 0; g.scolumn = 0;
    } else {
        q.G_max = gq->G_max; q.orth_max = gq->orth_max; q.value = gq->value; q.threshold = gq->threshold;
        q.n = gq->n; q.count_max = gq->count_max; q.column = gq->column; q.step = gq->step; q.code = gq->code;
        const GALIState<4>& G = gg->g;
        const SALIState& S = gg->s;
        g.gali[0] = G.gali[0]; g.gali[1] = G.gali[1]; g.gali[2] = G.gali[2]; g.gvalue = G.value; g.gn = G.n;
        g.gstep = G.step; g.gcode = G.code; g.gcolumn = G.column;
        g.svalue = S.value; g.sali = S.sali; g.sn = S.n; g.sstep = S.step; g.scode = S.code; g.scolumn = S.column;
        code0 = a.code[0][i];
        code1 = a.code[1][i];
        hstep0 = a.hstep[0] ? a.hstep[0][i] : 0;
        hstep1 = a.hstep[1] ? a.hstep[1][i] : 0;
    }
#pragma unroll
    for (int c = 0; c < 4; ++c) { q.lp[c] = split::LogProd{1.0, 0, 0}; g.lp[c] = split::LogProd{1.0, 0, 0}; }
    g.pending = 0;
    bool alive0 = code0 == STATUS_OK, alive1 = code1 == STATUS_OK;
    if (!alive0 && !alive1) return;   // frozen since an earlier launch: nothing is rewritten
    const double orth_tol = a.prm[0][0].orthogonality_tol;

    i64 n = a.n0;
    const i64 handoffs = a.steps / a.tau;
    for (i64 h = 0; h < handoffs; ++h) {
        if (alive0 && alive1) {   // the common case: one uniform test per window, not per step
            for (int t = 0; t < a.tau; ++t) {
                split::Jac J;
                split::jac(sys.nu, sys.kappa, sys.mu, x, J);
                split::apply32<K>(J, W0);
                split::apply64<K>(J, W1);
                split::forward(sys.nu, sys.kappa, sys.mu, x, J);
            }
        } else {
            for (int t = 0; t < a.tau; ++t) {
                split::Jac J;
                split::jac(sys.nu, sys.kappa, sys.mu, x, J);
                if (alive0) split::apply32<K>(J, W0);
                if (alive1) split::apply64<K>(J, W1);
                split::forward(sys.nu, sys.kappa, sys.mu, x, J);
            }
        }
        n += a.tau;
        const bool xok = finite_x(x);
        if (alive0) {   // _status (orbit.jl:3), then the chain, then _any_failed (orbit.jl:54-57)
            int8_t c = xok ? (finite32(W0) ? STATUS_OK : STATUS_W) : STATUS_STATE;
            if (c == STATUS_OK) {
                // the factorisation runs in the frame's registers: a failing handoff leaves the frame as it was
#pragma unroll
                for (int l = 0; l < 16; ++l) park_w[l] = W0[l];
                split::qr_handoff(q, n, W0, orth_tol);
                if (q.code != 0) {
                    c = STATUS_REDUCER;
#pragma unroll
                    for (int l = 0; l < 16; ++l) W0[l] = park_w[l];
                }
            }
            if (c != STATUS_OK) { code0 = c; hstep0 = n; alive0 = false; }
        }
        if (alive1) {
            int8_t c = xok ? (finite64(W1) ? STATUS_OK : STATUS_W) : STATUS_STATE;
            if (c == STATUS_OK) {
                // park the point and the Float32 frame in shared memory for the handoff (the clobber makes the
                // compiler reload them afterwards instead of keeping them in registers)
#pragma unroll
                for (int l = 0; l < 4; ++l) park_x[l] = x[l];
#pragma unroll
                for (int l = 0; l < 16; ++l) park_w[l] = W0[l];
                asm volatile("" ::: "memory");
                // the unit columns of a successful handoff go to the frame's output, where the values are formed
                // from them once, after the loop (the last successful handoff's are the ones the state keeps)
                if (split::gali_step(g, n, W1)) store_frame(a, 1, i, W1);
                asm volatile("" ::: "memory");
#pragma unroll
                for (int l = 0; l < 4; ++l) x[l] = park_x[l];
#pragma unroll
                for (int l = 0; l < 16; ++l) W0[l] = park_w[l];
                if (g.gcode != 0 || g.scode != 0) c = STATUS_REDUCER;
            }
            if (c != STATUS_OK) { code1 = c; hstep1 = n; alive1 = false; }
        }
        if (!alive0 && !alive1) break;
    }
    // orbit.jl:58: the final status check runs only at step N
    const bool xok = finite_x(x);
    if (alive0) { code0 = n == a.N ? (xok ? (finite32(W0) ? STATUS_OK : STATUS_W) : STATUS_STATE) : STATUS_OK; hstep0 = n; }
    if (alive1) { code1 = n == a.N ? (xok ? (finite64(W1) ? STATUS_OK : STATUS_W) : STATUS_STATE) : STATUS_OK; hstep1 = n; }

#pragma unroll
    for (int c = 0; c < 4; ++c) a.x_out[i * xso + c * xsc] = x[c];
    const bool was0 = fresh || a.code[0][i] == STATUS_OK, was1 = fresh || a.code[1][i] == STATUS_OK;
    if (g.pending) {   // GALI's and SALI's values of the last successful handoff of this launch
        double U[16];
        load_stored64(a, 1, i, U);
        split::gali_values(g, U);
    }
    if (was0) store_frame(a, 0, i, W0);
    if (was1) store_frame(a, 1, i, W1);
    // the records, one logarithm at a time (the frames are stored, so this tail needs few registers)
    if (was0) {
        QRState<4>* o = reinterpret_cast<QRState<4>*>(a.states[0] + i * QWORDS);
#pragma unroll 1
        for (int c = 0; c < 4; ++c) {
            CS s = fresh ? CS{0.0, 0.0} : gq->sums[c];
            split::lp_flush(s, q.lp[c]);
            o->sums[c] = s;
        }
        o->n = q.n; o->G_max = q.G_max; o->orth_max = q.orth_max; o->count_max = q.count_max;
        o->code = static_cast<int8_t>(q.code); o->column = q.column; o->value = q.value; o->threshold = q.threshold;
        o->step = q.step;
        a.code[0][i] = code0;
        if (a.hstep[0]) a.hstep[0][i] = hstep0;
    }
    if (was1) {
        GALIFrameState<4, true>* o = reinterpret_cast<GALIFrameState<4, true>*>(a.states[1] + i * GWORDS);
        GALIState<4>& G = o->g;
#pragma unroll 1
        for (int c = 0; c < 4; ++c) {
            CS cs = fresh ? CS{0.0, 0.0} : CS{gg->g.s[c], gg->g.c[c]};
            split::lp_flush(cs, g.lp[c]);
            G.s[c] = cs.s;
            G.c[c] = cs.c;
        }
        G.gali[0] = g.gali[0]; G.gali[1] = g.gali[1]; G.gali[2] = g.gali[2];
        G.value = g.gvalue; G.n = g.gn; G.step = g.gstep; G.code = static_cast<int8_t>(g.gcode); G.column = g.gcolumn;
        SALIState& S = o->s;
        // the SALI run's sums are GALI's columns 1-2 at SALI's last successful handoff, which is GALI's (a SALI
        // failure is a column-1 or column-2 norm failure, which stops GALI at the same handoff)
        S.s1 = CS{G.s[0], G.c[0]};
        S.s2 = CS{G.s[1], G.c[1]};
        S.sali = g.sali; S.value = g.svalue; S.n = g.sn; S.step = g.sstep; S.code = static_cast<int8_t>(g.scode);
        S.column = static_cast<int8_t>(g.scolumn);
        a.code[1][i] = code1;
        if (a.hstep[1]) a.hstep[1][i] = hstep1;
    }
}

template <int REGS>
cudaError_t launch_split(const cl_run& run, const KArgs& a, const double*, cudaStream_t st, LaunchInfo* info) {
    const SysFroeschle sys = make_sys<SysFroeschle>(run, nullptr);
    auto k = split_frames_kernel<REGS>;
    const int block = SPLIT_BLOCK;
    const long long grid = (a.n + block - 1) / block;
    k<<<static_cast<unsigned>(grid), block, SLOT_BYTES * block, st>>>(a, sys);
    const cudaError_t e = cudaGetLastError();
    if (info) {
        cudaFuncAttributes at;
        if (cudaFuncGetAttributes(&at, k) == cudaSuccess) info->regs = at.numRegs;
        info->block = block;
        info->grid = static_cast<int>(grid);
    }
    return e;
}

cudaError_t launch_split_any(const cl_run& run, const KArgs& a, const double* A, cudaStream_t st, LaunchInfo* info,
                             int minb) {
    (void)minb;   // one variant: 128 registers, 4 warps per scheduler (budgets of 96 or 80 registers spill and
                  // ran 7 % and 20 % slower at 65536 x 2000)
    return launch_split<128>(run, a, A, st, info);
}

// key of run_key for FroeschleMap (kind 3), d = 4, precision CL_PREC_MIXED_IND64, frames QRSpectrum(HouseholderQR) k = 4
// and GALI + SALI k = 4
const Registrar reg_split("s3d4p2|k4:QR4|k4:GALI,SALI|", launch_split_any, 1u << 3);

}  // namespace
}  // namespace cl
