// cl_mlp.cu -- the tensor-core kernels of the learned screen: a BF16 x BF16 -> FP32 GEMM on the 5th-generation
// tensor cores (tcgen05.mma, accumulator in tensor memory) with fused epilogues, and the elementwise kernels of the
// MLP's forward and backward passes (GELU, its derivative, the two-headed loss, bias gradients, Adam, transposes).
// No reference counterpart: the reference has no learned component.
//
// GEMM: C[M x N] = A[M x K] . B[N x K]^T (+ bias[N]) (+ C when accumulating), A and B row-major BF16 (K contiguous:
// both operands K-major). One CTA of 128 threads computes a 128 x NT tile (NT = 16..256) over its K range: a ring
// of 2-3 shared-memory stages, each a 128 x 64 block of A and an NT x 64 block of B in the canonical K-major
// no-swizzle layout (8-row x 16-byte core matrices, the two 8-element K halves of an MMA LBO = 128 B apart,
// consecutive 8-row groups SBO = 1024 B apart), filled by cp.async; one thread issues four tcgen05.mma (M = 128,
// N = NT, K = 16) per stage into an FP32 tile in tensor memory and commits them to the stage's mbarrier; after the
// last block each warp reads its 32 rows back with tcgen05.ld (warp w owns TMEM lanes 32w..32w+31) for the fused
// epilogue. Long-K products with few output tiles (weight gradients) split K over CTAs and add their partial tiles
// atomically. Every wait on an mbarrier is bounded: past the limit the kernel records an error flag and returns
// instead of spinning on.
#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <cstdio>
#include <string>

#include "../../include/chaoslab_b200.h"

namespace cl {

int capi_fail(int code, const std::string& msg);
int capi_map_cuda(cudaError_t e, const char* where);
void capi_count_launch();

namespace {

constexpr int BM = 128, BK = 64;
constexpr unsigned kWaitLimit = 1u << 26;   // mbarrier polls before giving up (a stuck MMA sets the flag)
constexpr uint64_t kWaitNs = 2000000000ull; // and at most 2 s of wall time per wait

__device__ unsigned g_mlp_error;            // nonzero after a bounded wait gave up

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// Shared-memory matrix descriptor (tcgen05): start >> 4 in bits 0-13, leading-dimension byte offset >> 4 in
// 16-29, stride-dimension byte offset >> 4 in 32-45, version 1 in 46-47, base offset 0, layout SWIZZLE_NONE (0).
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
    return (static_cast<uint64_t>((addr >> 4) & 0x3FFF)) | (static_cast<uint64_t>((lbo >> 4) & 0x3FFF) << 16) |
           (static_cast<uint64_t>((sbo >> 4) & 0x3FFF) << 32) | (1ull << 46);
}

// Instruction descriptor, kind::f16: FP32 accumulator (bits 4-5 = 1), BF16 A and B (bits 7-9, 10-12 = 1), both
// K-major (bits 15, 16 = 0), N >> 3 in bits 17-22, M >> 4 in bits 24-28.
__host__ __device__ constexpr uint32_t idesc_bf16(int M, int N) {
    return (1u << 4) | (1u << 7) | (1u << 10) | (static_cast<uint32_t>(N >> 3) << 17) | (static_cast<uint32_t>(M >> 4) << 24);
}

// Canonical K-major no-swizzle offset (bytes) of element (row, k) of a tile with 8 K-groups of 8 BF16 per block.
__device__ __forceinline__ uint32_t kmajor_off(int row, int k) {
    return static_cast<uint32_t>(((row >> 3) * (BK / 8) + (k >> 3)) * 128 + (row & 7) * 16 + (k & 7) * 2);
}

__device__ __forceinline__ uint64_t global_ns() {
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Waits for the mbarrier phase `phase`; gives up after kWaitLimit polls or kWaitNs nanoseconds, whichever first.
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t phase) {
    const uint64_t t0 = global_ns();
    for (unsigned it = 0; it < kWaitLimit; ++it) {
        uint32_t done;
        asm volatile(
            "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
            : "=r"(done) : "r"(bar), "r"(phase) : "memory");
        if (done) return true;
        if ((it & 255u) == 255u && global_ns() - t0 > kWaitNs) break;
    }
    atomicExch(&g_mlp_error, 1u);
    return false;
}

// The network's activation: GELU in its tanh form (Hendrycks & Gimpel 2016), x (1 + tanh u) / 2 with
// u = sqrt(2 / pi) (x + 0.044715 x^3). The forward pass (gelu_t, below) uses the special-function unit's tanh. The
// backward pass needs s = (1 + tanh u) / 2 = 1 / (1 + e^(-2u)) with its derivative, evaluated without the
// cancellation of 1 + tanh u for negative x as s = 1 / (1 + 2^z), z = -2 log2(e) u = x (G0 + G1 x^2) clamped to 64
// (beyond it s < 6e-20): one ex2 on the special-function unit, and the reciprocal on the FMA pipe from the seed
// bits(r0) = 0x7EF311C2 - bits(d), whose relative error is at most 0.0505 for every normal d (the constant
// minimises it over all mantissas; found by exhaustive search), refined by one Newton step r <- r + r t (error
// squared: 2.6e-3) and one third-order step r <- r + r (t + t^2) (error cubed: 1.7e-8), t = 1 - d r (run on -r,
// below); s is within 1.3 units in the last place (checked over 2e6 arguments).
constexpr float kG0 = -2.3022082f;     // -2 log2(e) sqrt(2 / pi)
constexpr float kG1 = -0.10294324f;    // kG0 * 0.044715
constexpr float kLn2 = 0.6931472f;
constexpr float kZMax = 64.0f;
constexpr uint32_t kRcpSeedNeg = 0xFEF311C2u;   // 0x7EF311C2 with the sign bit: the seed of -1 / d
__device__ __forceinline__ float ex2_approx(float z) {
    float e;
    asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(e) : "f"(z));
    return e;
}
// w = -1 / (1 + 2^z(x)) = -s for one value. The iteration runs on w ~ -1 / d so that its error term t = 1 + d w is
// one fused multiply-add of d itself (no negated copy of d): w <- w + w t (Newton), then w <- w + w (t + t^2); each
// operation is the exact negation of the same iteration on r ~ 1 / d, so -w is that iteration's s bit for bit.
__device__ __forceinline__ float negsig_t(float x) {
    const float z = fminf(__fmul_rn(x, __fmaf_rn(kG1, __fmul_rn(x, x), kG0)), kZMax);
    const float d = __fadd_rn(1.0f, ex2_approx(z));
    float w = __uint_as_float(kRcpSeedNeg - __float_as_uint(d));
    w = __fmaf_rn(w, __fmaf_rn(d, w, 1.0f), w);
    const float t = __fmaf_rn(d, w, 1.0f);
    return __fmaf_rn(w, __fmaf_rn(t, t, t), w);
}
__device__ __forceinline__ float sig_t(float x) { return -negsig_t(x); }
// The forward activation: (x / 2)(1 + tanh u), u = x (T0 + T1 x^2), with the special-function unit's tanh
// (tanh.approx.f32, relative error at most 2^-10.99): one special-function operation and four FP32 operations a
// value. Where tanh u is near -1 (x below about -2) the sum 1 + tanh u loses relative accuracy, but its absolute
// error stays below |x| 2^-12 (under 1e-3 for x > -4, and the value is ~0 beyond), smaller than the BF16 rounding
// of the activations the next layer adds it to.
constexpr float kT0 = 0.7978845608f;    // sqrt(2 / pi)
constexpr float kT1 = 0.0356774081f;    // sqrt(2 / pi) * 0.044715
__device__ __forceinline__ float tanh_approx(float u) {
    float t;
    asm("tanh.approx.f32 %0, %1;" : "=f"(t) : "f"(u));
    return t;
}
__device__ __forceinline__ float gelu_t(float x) {
    const float u = __fmul_rn(x, __fmaf_rn(kT1, __fmul_rn(x, x), kT0));
    const float h = __fmul_rn(x, 0.5f);
    return __fmaf_rn(h, tanh_approx(u), h);
}

// Packed FP32 pairs (the .f32x2 forms; lane by lane the same IEEE operations as the scalar ones).
__device__ __forceinline__ uint64_t f2(float a, float b) {
    uint64_t r;
    asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(a), "f"(b));
    return r;
}
__device__ __forceinline__ void f2split(uint64_t v, float& a, float& b) {
    asm("mov.b64 {%0, %1}, %2;" : "=f"(a), "=f"(b) : "l"(v));
}
__device__ __forceinline__ uint64_t fma2(uint64_t a, uint64_t b, uint64_t c) {
    uint64_t d;
    asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(d) : "l"(a), "l"(b), "l"(c));
    return d;
}
__device__ __forceinline__ uint64_t mul2(uint64_t a, uint64_t b) {
    uint64_t d;
    asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
    return d;
}
__device__ __forceinline__ uint64_t add2(uint64_t a, uint64_t b) {
    uint64_t d;
    asm("add.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
    return d;
}
// gelu_t of both lanes of v, rounded to a BF16 pair (low half: lane 0): the same operations lane by lane on packed
// FP32 pairs (fma/mul .f32x2), so the scalar form (the per-layer epilogue) and this one agree bit for bit.
__device__ __forceinline__ uint32_t gelu_t2_bf16(uint64_t v) {
    const uint64_t t1 = f2(kT1, kT1), t0 = f2(kT0, kT0), half = f2(0.5f, 0.5f);
    float u0, u1;
    f2split(mul2(v, fma2(t1, mul2(v, v), t0)), u0, u1);
    const uint64_t h = mul2(v, half);
    float y0, y1;
    f2split(fma2(h, f2(tanh_approx(u0), tanh_approx(u1)), h), y0, y1);
    const __nv_bfloat162 b = __floats2bfloat162_rn(y0, y1);
    return *reinterpret_cast<const uint32_t*>(&b);
}
// d/dx of the tanh-form GELU, s - x s (1 - s) ln2 (G0 + 3 G1 x^2) with s = 1 / (1 + 2^z) (the training's
// backward pass; the forward's tanh.approx differs from s by its rounding only).
__device__ __forceinline__ float gelu_t_grad(float x) {
    const float sg = sig_t(x);
    const float dz = __fmaf_rn(3.0f * kG1, __fmul_rn(x, x), kG0);
    return __fsub_rn(sg, __fmul_rn(__fmul_rn(__fmul_rn(x, sg), __fsub_rn(1.0f, sg)), __fmul_rn(kLn2, dz)));
}

// Async 16-byte global -> shared copy; src_bytes < 16 zero-fills the rest (0: nothing is read).
__device__ __forceinline__ void cp_async16(uint32_t dst, const void* src, uint32_t src_bytes) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" :: "r"(dst), "l"(src), "r"(src_bytes) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" :: "n"(N) : "memory"); }

// Stages one BM x BK (or NT x BK) block of a K-major BF16 matrix into the canonical no-swizzle layout. Chunk c of
// the tile (16 bytes = 8 elements) is row (c >> 6) * 8 + (c & 7), K-chunk (c >> 3) & 7: the 32 lanes of a warp
// cover 8 rows x 4 K-chunks, i.e. 64 contiguous bytes of each row in global memory and 8 distinct 16-byte bank
// groups in shared memory (4 wavefronts per 512 bytes, no conflicts).
template <int ROWS>
__device__ __forceinline__ void stage_tile(uint32_t dst, const __nv_bfloat16* __restrict__ G, int ld, int r0,
                                           int rows, int k0, int K, int tid) {
#pragma unroll
    for (int c = tid; c < ROWS * (BK / 8); c += 128) {
        const int r = (c >> 6) * 8 + (c & 7), kc = (c >> 3) & 7;
        const int gr = r0 + r, gk = k0 + kc * 8;
        const int valid = gr < rows ? max(0, min(8, K - gk)) : 0;
        const __nv_bfloat16* src = valid ? G + static_cast<size_t>(gr) * ld + gk : G;
        cp_async16(dst + kmajor_off(r, kc * 8), src, static_cast<uint32_t>(valid * 2));
    }
}

// C[M x N] (+)= A . B^T: one CTA of 128 threads per 128 x NT output tile and K range (split-K over gridDim.z).
// STAGES-deep ring of shared-memory stages filled by cp.async; one thread issues the stage's BK / 16 MMAs and
// commits them to the stage's mbarrier, which the copies into that stage wait on before it is refilled, so the
// loads of the next STAGES - 1 blocks overlap the tensor cores. With split-K (gridDim.z > 1) the partial tiles are
// added to C32 with atomics (C32 zeroed by the caller; no bias, epilogue or BF16 output).
template <int NT, int STAGES>
__global__ void __launch_bounds__(128, 1) gemm_bf16_tc(const __nv_bfloat16* __restrict__ A, int lda,
                                                       const __nv_bfloat16* __restrict__ B, int ldb, int M, int N,
                                                       int K, const float* __restrict__ bias, int epilogue,
                                                       float* __restrict__ C32, __nv_bfloat16* __restrict__ Cb,
                                                       int ldc, float* __restrict__ pre, int accumulate) {
    constexpr int TCOLS = NT < 32 ? 32 : NT;   // TMEM allocation: a power of two, at least 32 columns
    constexpr int A_BYTES = BM * BK * 2, B_BYTES = NT * BK * 2, STAGE_BYTES = A_BYTES + B_BYTES;
    static_assert((NT % 16) == 0 && NT >= 16 && NT <= 256, "N tile");
    extern __shared__ __align__(1024) uint8_t gsm[];
    __shared__ __align__(8) uint64_t mbar[STAGES];
    __shared__ uint32_t tmem_base;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int m0 = blockIdx.x * BM, n0 = blockIdx.y * NT;
    const int kblocks_all = (K + BK - 1) / BK;
    const int per = (kblocks_all + gridDim.z - 1) / gridDim.z;
    const int kb0 = blockIdx.z * per, kb1 = min(kblocks_all, kb0 + per), nkb = max(0, kb1 - kb0);
    const bool split = gridDim.z > 1;
    // vector epilogue: rows of C / pre start 32-byte aligned (ldc % 8 == 0 and 32-byte aligned bases)
    const bool vec = (ldc % 8) == 0 && (reinterpret_cast<uintptr_t>(C32) & 31) == 0 &&
                     (reinterpret_cast<uintptr_t>(Cb) & 15) == 0 && (reinterpret_cast<uintptr_t>(pre) & 31) == 0;

    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n"
                     :: "r"(smem_u32(&tmem_base)), "r"(TCOLS) : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::: "memory");
    }
    if (tid == 0) {
        for (int s = 0; s < STAGES; ++s)
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" :: "r"(smem_u32(&mbar[s])) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
    const uint32_t tmem = tmem_base;
    const uint32_t sbase = smem_u32(gsm);
    constexpr uint32_t idesc = idesc_bf16(BM, NT);
    bool ok = true;

    // prologue: the first STAGES - 1 blocks in flight (one commit group per block, empty past the end)
#pragma unroll
    for (int s = 0; s < STAGES - 1; ++s) {
        if (s < nkb) {
            const uint32_t st = sbase + s * STAGE_BYTES;
            stage_tile<BM>(st, A, lda, m0, M, (kb0 + s) * BK, K, tid);
            stage_tile<NT>(st + A_BYTES, B, ldb, n0, N, (kb0 + s) * BK, K, tid);
        }
        cp_async_commit();
    }
    int issued = -1;   // the last block whose MMAs were committed (thread 0 commits; the count is uniform)
    for (int i = 0; i < nkb && ok; ++i) {
        const int s = i % STAGES;
        cp_async_wait<STAGES - 2>();          // this thread's copies of block i have landed
        asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");   // visible to the tensor cores
        __syncthreads();                       // ... and every other thread's
        asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
        if (tid == 0) {
            const uint32_t st = sbase + s * STAGE_BYTES;
#pragma unroll
            for (int k = 0; k < BK / 16; ++k) {
                const uint64_t da = smem_desc(st + k * 256, 128, (BK / 8) * 128);
                const uint64_t db = smem_desc(st + A_BYTES + k * 256, 128, (BK / 8) * 128);
                const uint32_t acc = (i > 0 || k > 0) ? 1u : 0u;
                asm volatile(
                    "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
                    " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n"
                    :: "r"(tmem), "l"(da), "l"(db), "r"(idesc), "r"(acc) : "memory");
            }
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n"
                         :: "r"(smem_u32(&mbar[s])) : "memory");
        }
        issued = i;
        // refill the stage of block i - 1 with block i + STAGES - 1, once block i - 1's MMAs are done with it. Every
        // thread waits (bounded) and the CTA then agrees: one thread that gives up makes all of them leave the loop
        // at this same iteration, so every later barrier is reached by all threads.
        const int nx = i + STAGES - 1;
        if (nx < nkb) {   // uniform: i and nkb are the same in every thread
            bool w = true;
            if (i >= 1) {
                const int ps = (i - 1) % STAGES;
                w = mbar_wait(smem_u32(&mbar[ps]), static_cast<uint32_t>(((i - 1) / STAGES) & 1));
            }
            ok = __syncthreads_and(w) != 0;
            if (ok) {
                const uint32_t st = sbase + (nx % STAGES) * STAGE_BYTES;
                stage_tile<BM>(st, A, lda, m0, M, (kb0 + nx) * BK, K, tid);
                stage_tile<NT>(st + A_BYTES, B, ldb, n0, N, (kb0 + nx) * BK, K, tid);
            }
        }
        cp_async_commit();
    }
    cp_async_wait<0>();
    // The last committed block's barrier completes after every earlier MMA (they run in issue order). It is awaited
    // whether or not an earlier wait gave up, so the accumulator is neither read nor deallocated while an MMA that
    // was issued may still write it; a second give-up leaves the error flag set and the tile unwritten.
    {
        bool w = true;
        if (issued >= 0) w = mbar_wait(smem_u32(&mbar[issued % STAGES]), static_cast<uint32_t>((issued / STAGES) & 1));
        ok = __syncthreads_and(w && ok) != 0;
    }
    asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");

    if (ok && nkb > 0) {
        // epilogue: warp w reads TMEM lanes 32w..32w+31 (its rows), 16 columns at a time
        const int row = m0 + warp * 32 + lane;
#pragma unroll 1
        for (int c0 = 0; c0 < NT; c0 += 16) {
            uint32_t r[16];
            const uint32_t taddr = tmem + (static_cast<uint32_t>(warp * 32) << 16) + static_cast<uint32_t>(c0);
            asm volatile(
                "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];\n"
                : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
                  "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
                : "r"(taddr));
            asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
            if (row < M) {
                const int colb = n0 + c0;
                const size_t at0 = static_cast<size_t>(row) * ldc + colb;
                if (split) {
#pragma unroll
                    for (int j = 0; j < 16; ++j)
                        if (colb + j < N) atomicAdd(C32 + at0 + j, __uint_as_float(r[j]));
                } else if (vec && colb + 16 <= N) {
                    // a whole 16-column chunk: 16-byte loads and stores (rows 32-byte aligned: ldc % 8 == 0)
                    float v[16];
#pragma unroll
                    for (int j = 0; j < 16; ++j) v[j] = __uint_as_float(r[j]);
                    if (accumulate && C32) {
#pragma unroll
                        for (int q = 0; q < 4; ++q) {
                            const float4 c = reinterpret_cast<const float4*>(C32 + at0)[q];
                            v[4 * q] += c.x; v[4 * q + 1] += c.y; v[4 * q + 2] += c.z; v[4 * q + 3] += c.w;
                        }
                    }
                    if (bias) {
#pragma unroll
                        for (int j = 0; j < 16; ++j) v[j] += bias[colb + j];
                    }
                    if (pre) {
#pragma unroll
                        for (int q = 0; q < 4; ++q)
                            reinterpret_cast<float4*>(pre + at0)[q] = make_float4(v[4 * q], v[4 * q + 1], v[4 * q + 2], v[4 * q + 3]);
                    }
                    if (epilogue == 1) {
#pragma unroll
                        for (int j = 0; j < 16; ++j) v[j] = gelu_t(v[j]);
                    }
                    if (C32) {
#pragma unroll
                        for (int q = 0; q < 4; ++q)
                            reinterpret_cast<float4*>(C32 + at0)[q] = make_float4(v[4 * q], v[4 * q + 1], v[4 * q + 2], v[4 * q + 3]);
                    }
                    if (Cb) {
                        uint32_t w[8];
#pragma unroll
                        for (int q = 0; q < 8; ++q) {
                            const __nv_bfloat162 h = __floats2bfloat162_rn(v[2 * q], v[2 * q + 1]);
                            w[q] = *reinterpret_cast<const uint32_t*>(&h);
                        }
                        reinterpret_cast<uint4*>(Cb + at0)[0] = make_uint4(w[0], w[1], w[2], w[3]);
                        reinterpret_cast<uint4*>(Cb + at0)[1] = make_uint4(w[4], w[5], w[6], w[7]);
                    }
                } else {
#pragma unroll
                    for (int j = 0; j < 16; ++j) {
                        const int col = colb + j;
                        if (col >= N) continue;
                        float v = __uint_as_float(r[j]);
                        const size_t at = at0 + j;
                        if (accumulate && C32) v += C32[at];
                        if (bias) v += bias[col];
                        if (pre) pre[at] = v;
                        if (epilogue == 1) v = gelu_t(v);
                        if (C32) C32[at] = v;
                        if (Cb) Cb[at] = __float2bfloat16(v);
                    }
                }
            }
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
    __syncthreads();
    if (warp == 0) {
        asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" :: "r"(tmem), "r"(TCOLS) : "memory");
    }
}

// ---- the fused forward pass --------------------------------------------------------------------------------------
// The screen network's whole inference pass (64 -> 256 -> 256 -> 256 -> 16) in one persistent kernel, one CTA of
// eighteen warps per SM looping over 128-row tiles in pairs, the activations never leaving the SM. The two tiles of a
// pair sit in two slots, each with its activation tile in shared memory (64 KB; the input tile is copied into its
// last K block) and its 256-column FP32 accumulator in tensor memory (512 columns for both), and run ping-pong: the
// tensor cores compute one slot's layer while the epilogue drains the other slot's accumulator.
//   warp 0      producer: copies each tile's input by tensor-map TMA (eight 128-row x 8-column boxes landing as
//               K-major core matrices) and streams the weights through a 3-stage ring by bulk copies (cp.async.bulk)
//               from their pre-packed layout (cl_b200_mlp_pack_kmajor), each stage's mbarrier counting the bytes in;
//   warp 1      one thread issues the tcgen05.mma (M = 128, N = 256 / 16, K = 16 each) in the order slot 0, slot 1
//               per layer and commits them to the barriers that free a weight stage, a slot's input or hand an
//               accumulator to the epilogue;
//   warps 2..17 epilogue: read the accumulator (tcgen05.ld, the next 16 columns loading while the current ones are
//               processed), add the bias, apply GELU (packed FP32 pairs), round to BF16 into the slot's activation
//               tile, then release the slot to its next layer's MMAs.
// The MMAs see the operands in the same order as the per-layer GEMM (K ascending in steps of 16, accumulate from
// zero) and the epilogue is the same arithmetic, so the outputs are bit for bit the per-layer path's. Every wait is
// bounded: a wait that gives up sets the error flag and a shared abort flag that every role polls, all roles leave
// their loops, the MMA thread waits for its last commit and the producer for its copies in flight, then the
// accumulator is released.
constexpr int F_STAGES = 3;
constexpr int F_TILE = BM * BK * 2;                 // 16 KB: one 128 x 64 BF16 block (an input tile or activation block)
constexpr int F_SLOT = 4 * F_TILE;                  // 64 KB: one slot's activation tile, 4 K blocks of 64
constexpr int F_WCHUNK = 256 * BK * 2;              // 32 KB: one 256 x 64 weight block
constexpr int F_OFF_ACT = 0;                        // two slots
constexpr int F_OFF_W = F_OFF_ACT + 2 * F_SLOT;     // the weight ring
constexpr int F_SMEM = F_OFF_W + F_STAGES * F_WCHUNK;   // 229,376 bytes
constexpr int F_CHUNKS = 10;                        // per tile: W1 (1 block), W2 (4), W3 (4), W4 (its 4 blocks, 8 KB)
constexpr int F_THREADS = 576;                     // 18 warps: producer, MMA, 16 epilogue
constexpr int F_EPI_WARPS = 16;
constexpr int F_SLEEP_NS = 32;                     // the producer's and MMA issuer's poll interval

struct FusedArgs {
    const __nv_bfloat16* X;                         // B x 64 row-major, rows 16-byte aligned
    const uint8_t* Wp[4];                           // packed weights: 32 KB, 128 KB, 128 KB, 8 KB
    const float* bias[4];                           // 256, 256, 256, 16
    float* out;                                     // B x 16
    int B;
    int tiles;
};

__device__ __forceinline__ uint32_t fchunk_bytes(int c) { return c == F_CHUNKS - 1 ? 4u * 16 * BK * 2 : static_cast<uint32_t>(F_WCHUNK); }
__device__ __forceinline__ const uint8_t* fchunk_src(const FusedArgs& a, int c) {
    if (c == 0) return a.Wp[0];
    if (c <= 4) return a.Wp[1] + static_cast<size_t>(c - 1) * F_WCHUNK;
    if (c <= 8) return a.Wp[2] + static_cast<size_t>(c - 5) * F_WCHUNK;
    return a.Wp[3];
}

// Bounded wait that also gives up when another role has (the shared abort flag): the clock and the flag are
// checked every 64 polls. (A suspend-time hint on the try_wait made the kernel slower: 58.8 us against 51.1 us at
// 65536 rows.)
// SLEEP_NS > 0 (the single-thread roles: producer, MMA issuer) sleeps between polls, leaving the issue slots of its
// scheduler to the epilogue warps that share it.
template <int SLEEP_NS = 0>
__device__ __forceinline__ bool fwait(uint32_t bar, uint32_t parity, volatile int* abort_flag) {
    const uint64_t t0 = global_ns();
    for (unsigned it = 0;; ++it) {
        uint32_t done;
        asm volatile(
            "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
            : "=r"(done) : "r"(bar), "r"(parity) : "memory");
        if (done) return true;
        if (SLEEP_NS > 0) __nanosleep(SLEEP_NS);
        if ((it & 63u) == 63u) {
            if (*abort_flag) return false;
            if (it >= kWaitLimit || global_ns() - t0 > kWaitNs) {
                *abort_flag = 1;
                atomicExch(&g_mlp_error, 1u);
                return false;
            }
        }
    }
}

__device__ __forceinline__ void mbar_arrive(uint32_t bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];\n" :: "r"(bar) : "memory");
}

__device__ __forceinline__ void mma_commit(uint32_t bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" :: "r"(bar) : "memory");
}

__device__ __forceinline__ void mma_bf16(uint32_t tmem, uint64_t da, uint64_t db, uint32_t idesc, uint32_t acc) {
    asm volatile("{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
                 " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n"
                 :: "r"(tmem), "l"(da), "l"(db), "r"(idesc), "r"(acc) : "memory");
}

// 32 lanes x 16 columns of FP32 from tensor memory (no wait).
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, uint32_t (&r)[16]) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];\n"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
}

// Waits for this thread's tensor-memory loads; the registers pass through the wait so no use of them is scheduled
// before it.
__device__ __forceinline__ void tmem_wait16(uint32_t (&r)[16]) {
    asm volatile("tcgen05.wait::ld.sync.aligned;\n"
                 : "+r"(r[0]), "+r"(r[1]), "+r"(r[2]), "+r"(r[3]), "+r"(r[4]), "+r"(r[5]), "+r"(r[6]), "+r"(r[7]),
                   "+r"(r[8]), "+r"(r[9]), "+r"(r[10]), "+r"(r[11]), "+r"(r[12]), "+r"(r[13]), "+r"(r[14]), "+r"(r[15])
                 :: "memory");
}

__global__ void __launch_bounds__(F_THREADS, 1) mlp_forward_fused(const FusedArgs a, const __grid_constant__ CUtensorMap xmap) {
    extern __shared__ __align__(1024) uint8_t fsm[];
    __shared__ __align__(8) uint64_t w_full[F_STAGES], w_empty[F_STAGES], x_full[2], x_empty[2], acc_full[2],
        epi_done[2];
    __shared__ uint32_t tmem_base;
    __shared__ volatile int abort_flag;
    __shared__ int consumed_chunks, consumed_x;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const uint32_t sbase = smem_u32(fsm);
    const uint32_t sAct = sbase + F_OFF_ACT, sW = sbase + F_OFF_W;

    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n"
                     :: "r"(smem_u32(&tmem_base)), "r"(512) : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::: "memory");
    }
    if (tid == 0) {
        auto init = [](uint64_t* b, int count) {
            asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" :: "r"(smem_u32(b)), "r"(count) : "memory");
        };
        for (int s = 0; s < F_STAGES; ++s) { init(&w_full[s], 1); init(&w_empty[s], 1); }
        for (int s = 0; s < 2; ++s) {
            init(&x_full[s], 1); init(&x_empty[s], 1); init(&acc_full[s], 1); init(&epi_done[s], F_EPI_WARPS);
        }
        asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
        abort_flag = 0;
        consumed_chunks = 0;
        consumed_x = 0;
    }
    asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
    const uint32_t tmem = tmem_base;
    // this CTA's tiles k = 0, 1, ... (tile blockIdx.x + k gridDim.x) run in pairs: tile k in slot k & 1
    const int ntiles = a.tiles > static_cast<int>(blockIdx.x) ? (a.tiles - 1 - static_cast<int>(blockIdx.x)) / static_cast<int>(gridDim.x) + 1 : 0;
    const int npairs = (ntiles + 1) / 2;
    int issued_chunks = 0;        // producer: weight chunks whose copies were issued
    int issued_x = 0;             // producer: input tiles whose copies were issued
    int last_commit = -1;         // MMA thread: the last weight chunk whose MMAs were committed

    if (warp == 0) {
        // ---------------------------------------------------------------- producer (lane 0 issues)
        bool ok = true;
        int g = 0;
        for (int p = 0; p < npairs && ok; ++p)
            for (int l = 0; l < 4 && ok; ++l)
                for (int s = 0; s < 2 && ok; ++s) {
                    const int k = 2 * p + s;
                    if (k >= ntiles) continue;
                    int good = 1;
                    if (lane == 0) {
                        if (l == 0) {
                            // the 128 x 64 input tile into K block 3 of the slot's activation tile: eight tensor copies
                            // of 128 rows x 8 columns, K group g at g * 2048 bytes; rows past B are zero filled
                            good = fwait<F_SLEEP_NS>(smem_u32(&x_empty[s]), static_cast<uint32_t>((p & 1) ^ 1), &abort_flag);
                            if (good) {
                                const int tile = static_cast<int>(blockIdx.x) + k * static_cast<int>(gridDim.x);
                                const uint32_t bar = smem_u32(&x_full[s]), dst = sAct + s * F_SLOT + 3 * F_TILE;
                                asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" :: "r"(bar), "r"(F_TILE) : "memory");
#pragma unroll
                                for (int gk = 0; gk < 8; ++gk)
                                    asm volatile(
                                        "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];\n"
                                        :: "r"(dst + gk * 2048), "l"(reinterpret_cast<uint64_t>(&xmap)), "r"(gk * 8), "r"(tile * BM), "r"(bar)
                                        : "memory");
                                ++issued_x;
                            }
                        }
                        const int c_lo = l == 0 ? 0 : l == 1 ? 1 : l == 2 ? 5 : 9, c_hi = l == 0 ? 1 : l == 1 ? 5 : l == 2 ? 9 : 10;
                        for (int c = c_lo; c < c_hi && good; ++c, ++g) {
                            const int sw = g % F_STAGES;
                            good = fwait<F_SLEEP_NS>(smem_u32(&w_empty[sw]), static_cast<uint32_t>(((g / F_STAGES) & 1) ^ 1), &abort_flag);
                            if (!good) break;
                            const uint32_t bytes = fchunk_bytes(c), bar = smem_u32(&w_full[sw]);
                            asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" :: "r"(bar), "r"(bytes) : "memory");
                            asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n"
                                         :: "r"(sW + sw * F_WCHUNK), "l"(fchunk_src(a, c)), "r"(bytes), "r"(bar) : "memory");
                            ++issued_chunks;
                        }
                    }
                    ok = __shfl_sync(0xffffffffu, good, 0) != 0;
                }
    } else if (warp == 1) {
        // ---------------------------------------------------------------- MMA issuer (lane 0)
        // Order: per pair, per layer, slot 0 then slot 1, so one slot's MMAs run while the epilogue drains the
        // other slot's accumulator. A slot's layer l waits for its epilogue of layer l - 1 (the accumulator drained and
        // the activation tile written: epi_done, completion 4u + l - 1 for its u-th tile).
        if (lane == 0) {
            constexpr uint32_t id256 = idesc_bf16(BM, 256), id16 = idesc_bf16(BM, 16);
            bool ok = true;
            int g = 0, xw = 0;
            for (int p = 0; p < npairs && ok; ++p)
                for (int l = 0; l < 4 && ok; ++l)
                    for (int s = 0; s < 2 && ok; ++s) {
                        const int k = 2 * p + s;
                        if (k >= ntiles) continue;
                        ok = fwait<F_SLEEP_NS>(smem_u32(&epi_done[s]), static_cast<uint32_t>((4 * p + l - 1) & 1), &abort_flag);
                        if (ok && l == 0) {
                            ok = fwait<F_SLEEP_NS>(smem_u32(&x_full[s]), static_cast<uint32_t>(p & 1), &abort_flag);
                            if (ok) consumed_x = ++xw;
                        }
                        if (!ok) break;
                        asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
                        const uint32_t accum = tmem + static_cast<uint32_t>(s * 256);
                        const uint32_t act = sAct + s * F_SLOT;
                        const int nkb = l == 0 ? 1 : 4;
                        for (int kb = 0; kb < nkb && ok; ++kb) {
                            // layers 1-3: one weight chunk per K block; layer 4: one chunk holds all four blocks
                            const int sw = g % F_STAGES;
                            if (l != 3 || kb == 0)
                                ok = fwait<F_SLEEP_NS>(smem_u32(&w_full[sw]), static_cast<uint32_t>((g / F_STAGES) & 1), &abort_flag);
                            if (!ok) break;
                            asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
                            const uint32_t bbase = sW + sw * F_WCHUNK + (l == 3 ? kb * (16 * BK * 2) : 0);
                            // A: the input tile in the tensor copies' layout (LBO 2048, SBO 128) or an activation
                            // block in the epilogue's (LBO 128, SBO 1024)
                            const uint32_t abase = l == 0 ? act + 3 * F_TILE : act + kb * F_TILE;
                            const uint32_t astep = l == 0 ? 4096u : 256u, albo = l == 0 ? 2048u : 128u, asbo = l == 0 ? 128u : 1024u;
#pragma unroll
                            for (int kk = 0; kk < BK / 16; ++kk)
                                mma_bf16(accum, smem_desc(abase + kk * astep, albo, asbo),
                                         smem_desc(bbase + kk * 256, 128, (BK / 8) * 128), l == 3 ? id16 : id256,
                                         (kb > 0 || kk > 0) ? 1u : 0u);
                            if (l != 3) {
                                mma_commit(smem_u32(&w_empty[sw]));
                                last_commit = g;
                                ++g;
                            }
                        }
                        if (!ok) break;
                        if (l == 3) {
                            mma_commit(smem_u32(&w_empty[g % F_STAGES]));
                            last_commit = g;
                            ++g;
                            mma_commit(smem_u32(&x_empty[s]));   // the activation tile is free for the next input
                        }
                        mma_commit(smem_u32(&acc_full[s]));
                    }
            consumed_chunks = g;
        }
    } else {
        // ---------------------------------------------------------------- epilogue (warps 2..17)
        // warp w reads TMEM lanes 32 (w % 4) .. +31 (its rows); the four warps of a lane quarter split each 64-column
        // block into 16-column quarters h = (w - 2) / 4
        const int e = warp - 2, q = warp & 3, h = e >> 2;
        const int row = q * 32 + lane;
        bool ok = true;
        for (int p = 0; p < npairs && ok; ++p)
            for (int l = 0; l < 4 && ok; ++l)
                for (int s = 0; s < 2 && ok; ++s) {
                    const int k = 2 * p + s;
                    if (k >= ntiles) continue;
                    const int tile = static_cast<int>(blockIdx.x) + k * static_cast<int>(gridDim.x);
                    ok = __all_sync(0xffffffffu, fwait(smem_u32(&acc_full[s]), static_cast<uint32_t>(l & 1), &abort_flag));
                    if (!ok) break;
                    asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
                    const uint32_t tl = tmem + (static_cast<uint32_t>(q * 32) << 16) + static_cast<uint32_t>(s * 256);
                    if (l < 3) {
                        const float4* bias4 = reinterpret_cast<const float4*>(l == 0 ? a.bias[0] : l == 1 ? a.bias[1] : a.bias[2]);
                        const uint32_t act = sAct + s * F_SLOT;
                        uint32_t r[2][16];
                        tmem_ld16(tl + static_cast<uint32_t>(h * 16), r[0]);
                        tmem_wait16(r[0]);
#pragma unroll
                        for (int j = 0; j < 4; ++j) {
                            // the next block's load is in flight while this one is processed
                            if (j < 3) tmem_ld16(tl + static_cast<uint32_t>((j + 1) * 64 + h * 16), r[(j + 1) & 1]);
                            const uint32_t* v = r[j & 1];
                            const int c0 = j * 64 + h * 16;
                            uint32_t w8[8];
#pragma unroll
                            for (int pp = 0; pp < 4; ++pp) {
                                const float4 bb = __ldg(bias4 + (c0 >> 2) + pp);
                                const uint64_t v01 = add2(f2(__uint_as_float(v[4 * pp]), __uint_as_float(v[4 * pp + 1])), f2(bb.x, bb.y));
                                const uint64_t v23 = add2(f2(__uint_as_float(v[4 * pp + 2]), __uint_as_float(v[4 * pp + 3])), f2(bb.z, bb.w));
                                w8[2 * pp] = gelu_t2_bf16(v01);
                                w8[2 * pp + 1] = gelu_t2_bf16(v23);
                            }
                            const uint32_t blk = act + j * F_TILE;
                            asm volatile("st.shared.v4.b32 [%0], {%1, %2, %3, %4};\n"
                                         :: "r"(blk + kmajor_off(row, h * 16)), "r"(w8[0]), "r"(w8[1]), "r"(w8[2]), "r"(w8[3]) : "memory");
                            asm volatile("st.shared.v4.b32 [%0], {%1, %2, %3, %4};\n"
                                         :: "r"(blk + kmajor_off(row, h * 16 + 8)), "r"(w8[4]), "r"(w8[5]), "r"(w8[6]), "r"(w8[7]) : "memory");
                            if (j < 3) tmem_wait16(r[(j + 1) & 1]);
                        }
                        // the activation tile is written: visible to the tensor cores
                        asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
                    } else {
                        uint32_t r[4];
                        asm volatile("tcgen05.ld.sync.aligned.32x32b.x4.b32 {%0,%1,%2,%3}, [%4];\n"
                                     : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]) : "r"(tl + static_cast<uint32_t>(h * 4)));
                        asm volatile("tcgen05.wait::ld.sync.aligned;\n" : "+r"(r[0]), "+r"(r[1]), "+r"(r[2]), "+r"(r[3]) :: "memory");
                        const int grow = tile * BM + row;
                        if (grow < a.B) {
                            const float4 bb = __ldg(reinterpret_cast<const float4*>(a.bias[3]) + h);
                            reinterpret_cast<float4*>(a.out + static_cast<size_t>(grow) * 16)[h] =
                                make_float4(__fadd_rn(__uint_as_float(r[0]), bb.x), __fadd_rn(__uint_as_float(r[1]), bb.y),
                                            __fadd_rn(__uint_as_float(r[2]), bb.z), __fadd_rn(__uint_as_float(r[3]), bb.w));
                        }
                    }
                    // the accumulator is drained (and the activation tile written): the slot's next MMAs may start
                    asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
                    __syncwarp();
                    if (lane == 0) mbar_arrive(smem_u32(&epi_done[s]));
                }
    }
    __syncwarp();
    __syncthreads();
    // drain after an abort (nothing is outstanding on the normal path): the producer's copies in flight land, the
    // MMA thread's last commit completes, before the shared memory and the accumulator are released
    if (warp == 0 && lane == 0) {
        for (int g = consumed_chunks; g < issued_chunks; ++g) {
            int dummy = 0;
            fwait(smem_u32(&w_full[g % F_STAGES]), static_cast<uint32_t>((g / F_STAGES) & 1), reinterpret_cast<volatile int*>(&dummy));
        }
        for (int t = consumed_x; t < issued_x; ++t) {
            // input copy t went to slot (its tile index) & 1 as the slot's (t >> 1)-th use: the k-th tile of this CTA
            // has slot k & 1 and use k >> 1, and the copies were issued for k = 0, 1, 2, ...
            int dummy = 0;
            fwait(smem_u32(&x_full[t & 1]), static_cast<uint32_t>((t >> 1) & 1), reinterpret_cast<volatile int*>(&dummy));
        }
    }
    if (warp == 1 && lane == 0 && last_commit >= 0) {
        int dummy = 0;
        fwait(smem_u32(&w_empty[last_commit % F_STAGES]), static_cast<uint32_t>((last_commit / F_STAGES) & 1),
              reinterpret_cast<volatile int*>(&dummy));
    }
    asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
    __syncwarp();
    __syncthreads();
    if (warp == 0) {
        asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" :: "r"(tmem), "r"(512) : "memory");
    }
}

// Packs a row-major BF16 matrix (rows x cols, leading dimension ld) into tiles of `R` rows x 64 columns in the
// canonical K-major no-swizzle layout the MMAs read (zero padded to whole tiles): tile (rt, kb) is contiguous at
// (rt * nkb + kb) * R * 128 bytes. One thread per 16-byte chunk of the output.
__global__ void pack_kmajor(const __nv_bfloat16* __restrict__ src, int rows, int cols, int ld, int R, int nrt, int nkb,
                            __nv_bfloat16* __restrict__ dst) {
    const int64_t idx = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    const int64_t per_tile = static_cast<int64_t>(R) * 8;
    if (idx >= per_tile * nrt * nkb) return;
    const int64_t t = idx / per_tile;
    const int cc = static_cast<int>(idx % per_tile);
    const int rt = static_cast<int>(t / nkb), kb = static_cast<int>(t % nkb);
    const int r = rt * R + (cc >> 6) * 8 + (cc & 7), k0 = kb * 64 + ((cc >> 3) & 7) * 8;
    __nv_bfloat16 v[8];
#pragma unroll
    for (int j = 0; j < 8; ++j)
        v[j] = (r < rows && k0 + j < cols) ? src[static_cast<size_t>(r) * ld + k0 + j] : __float2bfloat16(0.f);
    uint4 w;
    memcpy(&w, v, 16);
    reinterpret_cast<uint4*>(dst)[idx] = w;
}

// ---- elementwise kernels ---------------------------------------------------------------------------------------------
__global__ void transpose_bf16(const __nv_bfloat16* __restrict__ src, int rows, int cols, int lds,
                               __nv_bfloat16* __restrict__ dst, int ldd) {
    __shared__ __nv_bfloat16 t[32][33];
    const int bx = blockIdx.x * 32, by = blockIdx.y * 32;
    for (int j = threadIdx.y; j < 32; j += blockDim.y) {
        const int r = by + j, c = bx + threadIdx.x;
        t[j][threadIdx.x] = (r < rows && c < cols) ? src[static_cast<size_t>(r) * lds + c] : __float2bfloat16(0.f);
    }
    __syncthreads();
    for (int j = threadIdx.y; j < 32; j += blockDim.y) {
        const int r = bx + j, c = by + threadIdx.x;   // dst is cols x rows
        if (r < cols && c < rows) dst[static_cast<size_t>(r) * ldd + c] = t[threadIdx.x][j];
    }
}

// dH = dY * GELU'(pre), written in BF16 for the next GEMMs and FP32 for the bias gradient.
__global__ void gelu_backward(const float* __restrict__ dY, const float* __restrict__ pre, int64_t n,
                              __nv_bfloat16* __restrict__ dHb, float* __restrict__ dH32) {
    const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float g = __fmul_rn(dY[i], gelu_t_grad(pre[i]));
    if (dHb) dHb[i] = __float2bfloat16(g);
    if (dH32) dH32[i] = g;
}

// Column sums of an FP32 matrix (bias gradients): db[j] = sum_i dH[i, j]. Blocks of 32 columns x 8 row lanes
// stride over the rows, fold their 8 partial sums in shared memory and add them to the (zeroed) output atomically,
// so the last bits of a sum depend on the order the blocks finish in.
__global__ void col_sum(const float* __restrict__ X, int rows, int cols, int ld, float* __restrict__ out) {
    __shared__ float part[8][33];
    const int j = blockIdx.x * 32 + threadIdx.x;
    float s = 0.f;
    if (j < cols)
        for (int i = blockIdx.y * 8 + threadIdx.y; i < rows; i += gridDim.y * 8) s += X[static_cast<size_t>(i) * ld + j];
    part[threadIdx.y][threadIdx.x] = s;
    __syncthreads();
    if (threadIdx.y == 0 && j < cols) {
        float t = part[0][threadIdx.x];
        for (int r = 1; r < 8; ++r) t += part[r][threadIdx.x];
        atomicAdd(out + j, t);
    }
}

// Head loss on logits [B x ld] (column 0: chaos logit, column 1: lambda_1 prediction): mean binary cross-entropy
// plus w_reg times the mean squared error; the gradient dL/dlogits (columns 0, 1; zero elsewhere), FP32 and BF16,
// and the per-row losses.
__global__ void head_loss(const float* __restrict__ logits, int B, int ld, const float* __restrict__ label,
                          const float* __restrict__ target, float w_reg, float* __restrict__ grad,
                          __nv_bfloat16* __restrict__ gradb, float* __restrict__ row_loss) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= B) return;
    const float z = logits[static_cast<size_t>(i) * ld], y = label[i];
    const float p = 1.0f / (1.0f + __expf(-z));
    const float bce = fmaxf(z, 0.f) - z * y + log1pf(__expf(-fabsf(z)));
    const float e = logits[static_cast<size_t>(i) * ld + 1] - target[i];
    row_loss[i] = bce + w_reg * e * e;
    for (int j = 0; j < ld; ++j) {
        float g = 0.f;
        if (j == 0) g = (p - y) / B;
        else if (j == 1) g = 2.0f * w_reg * e / B;
        grad[static_cast<size_t>(i) * ld + j] = g;
        if (gradb) gradb[static_cast<size_t>(i) * ld + j] = __float2bfloat16(g);
    }
}

// Adam on FP32 master weights; refreshes the BF16 copy (and its transpose when given: W is rows x cols).
__global__ void adam_step(float* __restrict__ w, const float* __restrict__ g, float* __restrict__ m,
                          float* __restrict__ v, int64_t n, float lr, float b1, float b2, float eps, float c1,
                          float c2, __nv_bfloat16* __restrict__ wb, __nv_bfloat16* __restrict__ wbt, int rows, int cols) {
    const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.0f - b1) * gi, vi = b2 * v[i] + (1.0f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    const float wi = w[i] - lr * (mi / c1) / (sqrtf(vi / c2) + eps);
    w[i] = wi;
    if (wb) wb[i] = __float2bfloat16(wi);
    if (wbt) {
        const int r = static_cast<int>(i / cols), c = static_cast<int>(i % cols);
        wbt[static_cast<size_t>(c) * rows + r] = __float2bfloat16(wi);
    }
}

// Screening features from the reducer states of the chain (MEGNO(replace = false), SALI()) on a k = 2 frame, Julia
// layout (MEGNOState 200 bytes, then SALIState 72 bytes, per orbit), read after the window ending at global step n:
// feature 3w + 0: log-stretch rate of column 1, (s + c) / n; 3w + 1: log10(max(SALI, 1e-16)) / 8; 3w + 2: the running
// MEGNO Y = 2 R1 / n of column 1, / 4. After the last window (w = windows - 1) also 60: the mean MEGNO Ybar / 4,
// 61: the log-stretch rate of column 2, 62: log10 SALI / 8 again, 63: 0.
__global__ void screen_features(const double* __restrict__ st, int64_t n_orbits, int64_t n, int w, int windows,
                                float* __restrict__ f32, __nv_bfloat16* __restrict__ fb) {
    const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= n_orbits) return;
    const double* s = st + i * 34;       // 272 bytes
    // MEGNOState: c1 {s, R1, R2, Q, Q2} (10 doubles), c2 (10), value, n, K, step, code|column
    const double tn = static_cast<double>(n);
    const double rate1 = (s[0] + s[1]) / tn, Y = 2.0 * (s[2] + s[3]) / tn;
    const double* sali = s + 25;         // SALIState: s1 (2), s2 (2), sali, ...
    const double lsal = log10(fmax(sali[4], 1e-16)) / 8.0;
    float v[3] = {static_cast<float>(rate1), static_cast<float>(lsal), static_cast<float>(Y / 4.0)};
    for (int j = 0; j < 3; ++j) {
        const int64_t at = i * 64 + 3 * w + j;
        if (f32) f32[at] = v[j];
        if (fb) fb[at] = __float2bfloat16(v[j]);
    }
    if (w == windows - 1) {
        const long long Kh = *reinterpret_cast<const long long*>(s + 22);
        const double Ybar = Kh > 0 ? (s[6] + s[7]) / static_cast<double>(Kh) : 0.0;
        const double rate2 = (s[10] + s[11]) / tn;
        float e[4] = {static_cast<float>(Ybar / 4.0), static_cast<float>(rate2), static_cast<float>(lsal), 0.f};
        for (int j = 0; j < 4; ++j) {
            const int64_t at = i * 64 + 60 + j;
            if (f32) f32[at] = e[j];
            if (fb) fb[at] = __float2bfloat16(e[j]);
        }
    }
}

__global__ void f32_to_bf16(const float* __restrict__ x, int64_t n, __nv_bfloat16* __restrict__ y) {
    const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i < n) y[i] = __float2bfloat16(x[i]);
}

template <int NT>
cudaError_t launch_gemm(const void* A, int lda, const void* B, int ldb, int M, int N, int K, const float* bias,
                        int epi, float* C32, void* Cb, int ldc, float* pre, int acc, int splits, cudaStream_t st) {
    // two CTAs per SM (one's epilogue overlaps the other's main loop): 96 KB of stages at NT = 256 and 128
    constexpr int STAGES = NT >= 256 ? 2 : 3;
    constexpr int smem = STAGES * (BM + NT) * BK * 2;
    auto k = gemm_bf16_tc<NT, STAGES>;
    // the attribute belongs to the current device's context: set before every launch (cheap and idempotent)
    const cudaError_t ea = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    if (ea != cudaSuccess) return ea;
    dim3 grid((M + BM - 1) / BM, (N + NT - 1) / NT, splits);
    k<<<grid, 128, smem, st>>>(static_cast<const __nv_bfloat16*>(A), lda, static_cast<const __nv_bfloat16*>(B), ldb,
                               M, N, K, bias, epi, C32, static_cast<__nv_bfloat16*>(Cb), ldc, pre, acc);
    return cudaGetLastError();
}

}  // namespace
}  // namespace cl

using namespace cl;

extern "C" {

int cl_b200_gemm_bf16(const void* A, int32_t lda, const void* B, int32_t ldb, int32_t M, int32_t N, int32_t K,
                      const float* bias, int32_t epilogue, float* C32, void* Cbf16, int32_t ldc, float* pre,
                      int32_t accumulate, void* stream) {
    if (!A || !B || M <= 0 || N <= 0 || K <= 0 || (!C32 && !Cbf16) || ldc < N)
        return capi_fail(CL_EINVAL, "gemm: bad arguments");
    if ((lda % 8) || (ldb % 8) || lda < K || ldb < K || (reinterpret_cast<uintptr_t>(A) % 16) ||
        (reinterpret_cast<uintptr_t>(B) % 16))
        return capi_fail(CL_EINVAL, "gemm: operands need 16-byte aligned rows (ld a multiple of 8, at least K)");
    if (epilogue != 0 && epilogue != 1) return capi_fail(CL_EINVAL, "gemm: epilogue 0 (none) or 1 (GELU)");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const int nt = N <= 16 ? 16 : N <= 64 ? 64 : N <= 128 ? 128 : 256;
    // split-K when the output tiles cannot fill the GPU and K is long (weight gradients: K = the batch); only
    // for a plain FP32 result, which the partial tiles are added into
    const int64_t tiles = static_cast<int64_t>((M + BM - 1) / BM) * ((N + nt - 1) / nt);
    const int kblocks = (K + BK - 1) / BK;
    int splits = 1;
    if (C32 && !Cbf16 && !bias && !pre && epilogue == 0 && tiles < 148 && kblocks >= 16) {
        splits = static_cast<int>(std::min<int64_t>(kblocks / 8, (2 * 148 + tiles - 1) / tiles));
        splits = std::max(1, std::min(splits, 1024));
        // the partial sums start from zero, or from C when accumulating
        if (!accumulate) {
            const cudaError_t e = cudaMemset2DAsync(C32, sizeof(float) * static_cast<size_t>(ldc), 0,
                                                    sizeof(float) * static_cast<size_t>(N), static_cast<size_t>(M), st);
            if (e != cudaSuccess) return capi_map_cuda(e, "gemm zero");
        }
    }
    cudaError_t e;
    if (nt == 16) e = launch_gemm<16>(A, lda, B, ldb, M, N, K, bias, epilogue, C32, Cbf16, ldc, pre, accumulate, splits, st);
    else if (nt == 64) e = launch_gemm<64>(A, lda, B, ldb, M, N, K, bias, epilogue, C32, Cbf16, ldc, pre, accumulate, splits, st);
    else if (nt == 128) e = launch_gemm<128>(A, lda, B, ldb, M, N, K, bias, epilogue, C32, Cbf16, ldc, pre, accumulate, splits, st);
    else e = launch_gemm<256>(A, lda, B, ldb, M, N, K, bias, epilogue, C32, Cbf16, ldc, pre, accumulate, splits, st);
    capi_count_launch();
    return e == cudaSuccess ? 0 : capi_map_cuda(e, "gemm launch");
}

// The input's tensor map: X (B x 64 BF16, rows of 128 bytes) as a 2D tensor, boxes of 8 columns x 128 rows, no
// swizzle, zero fill past row B. cuTensorMapEncodeTiled is the driver's; it is reached through the runtime's entry
// point query so the library links against the runtime alone.
static int encode_x_map(CUtensorMap* m, const void* X, int32_t B) {
    using Encode = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
    // looked up once per process (a function-local static: thread-safe initialisation); null if unavailable
    static const Encode enc = []() -> Encode {
        void* fn = nullptr;
        cudaDriverEntryPointQueryResult q;
        const cudaError_t e = cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q);
        return (e == cudaSuccess && q == cudaDriverEntryPointSuccess) ? reinterpret_cast<Encode>(fn) : nullptr;
    }();
    if (!enc) return cl::capi_fail(CL_EUNSUPPORTED, "fused forward: cuTensorMapEncodeTiled unavailable");
    const cuuint64_t dims[2] = {64, static_cast<cuuint64_t>(B)};
    const cuuint64_t strides[1] = {128};
    const cuuint32_t box[2] = {8, 128};
    const cuuint32_t estr[2] = {1, 1};
    const CUresult r = enc(m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<void*>(X), dims, strides, box, estr,
                           CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_NONE,
                           CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) return cl::capi_fail(CL_EINVAL, "fused forward: input tensor map rejected");
    return 0;
}

int cl_b200_mlp_pack_kmajor(const void* src, int32_t rows, int32_t cols, int32_t ld, int32_t tile_rows, void* dst,
                            void* stream) {
    if (!src || !dst || rows <= 0 || cols <= 0 || ld < cols || tile_rows <= 0 || (tile_rows % 8) != 0)
        return capi_fail(CL_EINVAL, "pack: bad arguments (tile_rows a positive multiple of 8)");
    if (reinterpret_cast<uintptr_t>(dst) % 16) return capi_fail(CL_EINVAL, "pack: dst needs 16-byte alignment");
    const int nrt = (rows + tile_rows - 1) / tile_rows, nkb = (cols + 63) / 64;
    const int64_t n = static_cast<int64_t>(tile_rows) * 8 * nrt * nkb;
    pack_kmajor<<<static_cast<unsigned>((n + 255) / 256), 256, 0, static_cast<cudaStream_t>(stream)>>>(
        static_cast<const __nv_bfloat16*>(src), rows, cols, ld, tile_rows, nrt, nkb, static_cast<__nv_bfloat16*>(dst));
    capi_count_launch();
    const cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? 0 : capi_map_cuda(e, "pack launch");
}

int cl_b200_mlp_forward_fused(const void* X, int32_t B, const void* Wp1, const void* Wp2, const void* Wp3,
                              const void* Wp4, const float* b1, const float* b2, const float* b3, const float* b4,
                              float* out, int32_t max_ctas, void* stream) {
    if (!X || !Wp1 || !Wp2 || !Wp3 || !Wp4 || !b1 || !b2 || !b3 || !b4 || !out || B <= 0 || max_ctas < 0)
        return capi_fail(CL_EINVAL, "fused forward: bad arguments");
    const void* ps[10] = {X, Wp1, Wp2, Wp3, Wp4, out, b1, b2, b3, b4};
    for (const void* p : ps)
        if (reinterpret_cast<uintptr_t>(p) % 16) return capi_fail(CL_EINVAL, "fused forward: X, the packed weights, the biases and out need 16-byte alignment");
    int dev = 0, sms = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(mlp_forward_fused, cudaFuncAttributeMaxDynamicSharedMemorySize, F_SMEM);
    if (e != cudaSuccess) return capi_map_cuda(e, "fused forward setup");
    FusedArgs a;
    a.X = static_cast<const __nv_bfloat16*>(X);
    a.Wp[0] = static_cast<const uint8_t*>(Wp1);
    a.Wp[1] = static_cast<const uint8_t*>(Wp2);
    a.Wp[2] = static_cast<const uint8_t*>(Wp3);
    a.Wp[3] = static_cast<const uint8_t*>(Wp4);
    a.bias[0] = b1; a.bias[1] = b2; a.bias[2] = b3; a.bias[3] = b4;
    a.out = out;
    a.B = B;
    a.tiles = (B + BM - 1) / BM;
    int grid = a.tiles < sms ? a.tiles : sms;
    if (max_ctas > 0 && grid > max_ctas) grid = max_ctas;
    CUtensorMap xmap;
    if (int rc = encode_x_map(&xmap, X, B)) return rc;
    mlp_forward_fused<<<static_cast<unsigned>(grid), F_THREADS, F_SMEM, static_cast<cudaStream_t>(stream)>>>(a, xmap);
    capi_count_launch();
    e = cudaGetLastError();
    return e == cudaSuccess ? 0 : capi_map_cuda(e, "fused forward launch");
}

int cl_b200_mlp_status(void) {
    unsigned v = 0;
    if (cudaMemcpyFromSymbol(&v, g_mlp_error, sizeof v) != cudaSuccess) return CL_EDEVICE_LOST;
    return v ? CL_EDEVICE_LOST : 0;
}

int cl_b200_transpose_bf16(const void* src, int32_t rows, int32_t cols, int32_t lds, void* dst, int32_t ldd, void* stream) {
    dim3 grid((cols + 31) / 32, (rows + 31) / 32), block(32, 8);
    transpose_bf16<<<grid, block, 0, static_cast<cudaStream_t>(stream)>>>(
        static_cast<const __nv_bfloat16*>(src), rows, cols, lds, static_cast<__nv_bfloat16*>(dst), ldd);
    const cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? 0 : capi_map_cuda(e, "transpose");
}

int cl_b200_gelu_backward(const float* dY, const float* pre, int64_t n, void* dHb, float* dH32, void* stream) {
    gelu_backward<<<static_cast<unsigned>((n + 255) / 256), 256, 0, static_cast<cudaStream_t>(stream)>>>(
        dY, pre, n, static_cast<__nv_bfloat16*>(dHb), dH32);
    const cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? 0 : capi_map_cuda(e, "gelu backward");
}

int cl_b200_col_sum(const float* X, int32_t rows, int32_t cols, int32_t ld, float* out, void* stream) {
    if (!X || !out || rows < 0 || cols <= 0 || ld < cols) return capi_fail(CL_EINVAL, "column sums: bad arguments");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    cudaError_t e = cudaMemsetAsync(out, 0, sizeof(float) * static_cast<size_t>(cols), st);
    if (e != cudaSuccess) return capi_map_cuda(e, "column sums");
    const unsigned gy = static_cast<unsigned>(std::min(1024, std::max(1, (rows + 255) / 256)));
    col_sum<<<dim3((cols + 31) / 32, gy), dim3(32, 8), 0, st>>>(X, rows, cols, ld, out);
    e = cudaGetLastError();
    return e == cudaSuccess ? 0 : capi_map_cuda(e, "column sums");
}

int cl_b200_head_loss(const float* logits, int32_t B, int32_t ld, const float* label, const float* target, float w_reg,
                      float* grad, void* gradb, float* row_loss, void* stream) {
    head_loss<<<(B + 127) / 128, 128, 0, static_cast<cudaStream_t>(stream)>>>(
        logits, B, ld, label, target, w_reg, grad, static_cast<__nv_bfloat16*>(gradb), row_loss);
    const cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? 0 : capi_map_cuda(e, "head loss");
}

int cl_b200_adam(float* w, const float* g, float* m, float* v, int64_t n, float lr, float b1, float b2, float eps,
                 int32_t t, void* wb, void* wbt, int32_t rows, int32_t cols, void* stream) {
    const float c1 = 1.0f - powf(b1, static_cast<float>(t)), c2 = 1.0f - powf(b2, static_cast<float>(t));
    adam_step<<<static_cast<unsigned>((n + 255) / 256), 256, 0, static_cast<cudaStream_t>(stream)>>>(
        w, g, m, v, n, lr, b1, b2, eps, c1, c2, static_cast<__nv_bfloat16*>(wb), static_cast<__nv_bfloat16*>(wbt),
        rows, cols);
    const cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? 0 : capi_map_cuda(e, "adam");
}

int cl_b200_screen_features(const void* states, int64_t n_orbits, int64_t n, int32_t window, int32_t windows,
                            float* f32, void* fbf16, void* stream) {
    if (!states || n_orbits <= 0 || n <= 0 || window < 0 || window >= windows || 3 * windows + 4 > 64)
        return capi_fail(CL_EINVAL, "screen features: bad arguments");
    screen_features<<<static_cast<unsigned>((n_orbits + 127) / 128), 128, 0, static_cast<cudaStream_t>(stream)>>>(
        static_cast<const double*>(states), n_orbits, n, window, windows, f32, static_cast<__nv_bfloat16*>(fbf16));
    const cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? 0 : capi_map_cuda(e, "screen features");
}

int cl_b200_to_bf16(const float* x, int64_t n, void* y, void* stream) {
    f32_to_bf16<<<static_cast<unsigned>((n + 255) / 256), 256, 0, static_cast<cudaStream_t>(stream)>>>(
        x, n, static_cast<__nv_bfloat16*>(y));
    const cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? 0 : capi_map_cuda(e, "to bf16");
}

}  // extern "C"
