// cl_coop.cuh -- the cooperative ensemble kernel for standard-map lattices (StandardMapChain, d = 2 NS >= 4): one
// orbit per group of G = NS lanes instead of one per thread, so the d x k frame no longer has to fit one thread's
// registers (at d = 16, k = 8 the one-thread kernel holds 128 frame entries and spills) and an orbit's step is
// spread over G lanes (a long orbit finishes G times sooner, which matters when the longest orbits set the time).
//
// Between handoffs lane j of a group owns lattice site j: its coordinates q_j, p_j (Float64) and rows j and NS + j of
// the frame (k entries each). A step is the reference's `tangent` at the old point, `ChainTangent * W` and `forward`
// (standard_map_chain.jl:38-60, chain_tangent.jl:53-91): each lane evaluates its own site's sine / cosine and its
// right bond's, and takes the left bond's values and its neighbours' frame rows from the neighbouring lanes by warp
// shuffles. At a handoff the group stages the frame in shared memory and runs QRSpectrum(HouseholderQR)
// (householder.jl:19-80, qr_spectrum.jl:36-74) column-parallel: lane j owns columns j, j + G, ...; the owner of
// column c builds reflector c in shared memory, every lane applies it to its own columns and forms its own columns
// of Q. window_Gw (one lane) and orth_loss read R and Q from shared memory.
//
// Every entry is computed by the same operations, in the same order and type, as in the one-thread kernel: the
// band product's sums, every left-folded dot product and norm, the reflectors' zero rows. Only the lane doing the
// work changes, so the results are bit-identical to the one-thread kernel (and, in Float64, to the oracle).
// Maxima combined across lanes (orth_loss, the escape test) use operations whose result does not depend on order.
#pragma once

#include "cl_ensemble.cuh"

namespace cl {

// Shared-memory words of one orbit's handoff workspace (in Real): the staged frame (D x K), Q (D x K), the
// reflectors (D x NREF; afterwards window_Gw's scratch column) and R (K x K).
template <int D, int K>
struct CoopSmem {
    static constexpr int NREF = K < D ? K : K - 1;
    static constexpr int T = D * K, Q = D * K, U = (D * NREF > K ? D * NREF : K), R = K * K;
    static constexpr int words = T + Q + U + R;
};

template <int G>
__device__ __forceinline__ unsigned group_mask(int lane) {
    return G == 32 ? 0xffffffffu : (((1u << G) - 1u) << (lane & ~(G - 1)));
}

template <int G>
__device__ __forceinline__ bool group_all(unsigned mask, bool p) {
    return (__ballot_sync(mask, p) & mask) == mask;
}

template <typename T>
__device__ __forceinline__ T rv(const T* R0, int l, bool rescale, T m) { return rescale ? dv(R0[l], m) : R0[l]; }

// window_Gw (orthonormalize.jl:112-127) on R in shared memory, one column of R^{-1} at a time (scratch `ri`, K
// words): the same operations in the same order as the register version in cl_qr.cuh. The two Frobenius sums are
// independent left folds in column-major order, so folding the inverse column by column changes nothing.
template <int K, typename T>
__device__ __forceinline__ T window_Gw_sm(const T* R0, T* ri) {
    T m = fabs(R0[0]);
#pragma unroll 1
    for (int l = 1; l < K * K; ++l) m = mx(m, static_cast<T>(fabs(R0[l])));
    bool rescale = false;
    if constexpr (sizeof(T) == 8) rescale = (m > T(1e100) || m < T(1e-100)) && isfin(m) && m > T(0);
    T a = rv(R0, 0, rescale, m) * rv(R0, 0, rescale, m);
#pragma unroll 1
    for (int l = 1; l < K * K; ++l) a = a + rv(R0, l, rescale, m) * rv(R0, l, rescale, m);
    T b = T(0);
#pragma unroll 1
    for (int jc = 0; jc < K; ++jc) {
#pragma unroll 1
        for (int i = 0; i < K; ++i) ri[i] = T(0);
        ri[jc] = dv(T(1), rv(R0, jc + jc * K, rescale, m));
#pragma unroll 1
        for (int i = jc - 1; i >= 0; --i) {
            T s = T(0);
#pragma unroll 1
            for (int l = i + 1; l <= jc; ++l) s = s + rv(R0, i + l * K, rescale, m) * ri[l];
            ri[i] = dv(-s, rv(R0, i + i * K, rescale, m));
        }
#pragma unroll 1
        for (int i = 0; i < K; ++i) b = (jc == 0 && i == 0) ? ri[0] * ri[0] : b + ri[i] * ri[i];
    }
    return sqt(a) * sqt(b);
}

// One lane's part of QRState<K>: the sums of its own columns; the scalars are kept identical in every lane.
template <int K, int KPL>
struct CoopQR {
    CS sums[KPL];
    i64 n, count_max, column, step;
    double G_max, orth_max, value, threshold;
    int8_t code;
};

// One lane's lattice site: its coordinates and its two rows of the frame, and the step of the chain on them. The
// group has G >= NS lanes (shuffle width G); lanes past the lattice (j >= NS) step a dummy site with no bonds.
template <int NS, typename Real, int K, int G = NS>
struct CoopSite {
    double q, p;
    Real Wq[K], Wp[K];

    // tangent at the old point (chain_tangent.jl:84-91): this site and its right bond; the left bond's values from
    // the left neighbour. ChainTangent * W (chain_tangent.jl:62-78) on rows j and NS + j of every column, with the
    // neighbours' rows by shuffles. forward (standard_map_chain.jl:38-44): p' = p + (K sin q + eps s), s = (0 +
    // sin(q_j - q_left)) + sin(q_j - q_right); q' = q + p'.
    __device__ __forceinline__ void step(unsigned gm, int jl, int jr, bool hasL, bool hasR, double Kc, double eps) {
        const double qr_ = __shfl_sync(gm, q, jr, G);
        double sb = 0.0, sq;
        Real g, gl, gr;
        if constexpr (sizeof(Real) == 4) {
            float cbf = 0.0f, cqf;
            if (hasR) {
                const Reduced w = cl_reduce(q - qr_);
                sb = cl_sin_split(w);
                float sf; cl_sincos32(w, &sf, &cbf);
            }
            const Reduced w = cl_reduce(q);
            sq = cl_sin_split(w);
            float sf; cl_sincos32(w, &sf, &cqf);
            const float cbfl = __shfl_sync(gm, cbf, jl, G);
            const float e = static_cast<float>(eps);
            const float cl_ = hasL ? e * cbfl : 0.0f, cr = hasR ? e * cbf : 0.0f;
            g = (static_cast<float>(Kc) * cqf + cl_) + cr;
            gl = -cl_;
            gr = -cr;
        } else {
            double cb = 0.0, cq;
            if (hasR) cl_sincos(q - qr_, &sb, &cb);
            cl_sincos(q, &sq, &cq);
            const double cbl = __shfl_sync(gm, cb, jl, G);
            const double cl_ = hasL ? eps * cbl : 0.0, cr = hasR ? eps * cb : 0.0;
            g = (Kc * cq + cl_) + cr;
            gl = -cl_;
            gr = -cr;
        }
        const double sbl = __shfl_sync(gm, sb, jl, G);
#pragma unroll
        for (int c = 0; c < K; ++c) {
            const Real wl = __shfl_sync(gm, Wq[c], jl, G), wr = __shfl_sync(gm, Wq[c], jr, G);
            Real t = g * Wq[c];
            if (hasL) t = t + gl * wl;
            if (hasR) t = t + gr * wr;
            const Real wq = Wq[c], wp = Wp[c];
            Wq[c] = (wq + t) + wp;
            Wp[c] = t + wp;
        }
        double s = 0.0;
        if (hasL) s = s + (-sbl);
        if (hasR) s = s + sb;
        p = p + (Kc * sq + eps * s);
        q = q + p;
    }
};

template <int NS, typename Real, int K, int TAU_UNROLL, int MINB>
__global__ void __launch_bounds__(128, MINB) coop_kernel(const EArgs a, const SysChain<NS> sys0) {
    constexpr int G = NS, D = 2 * NS, S = 2 * NS, KPL = K / G;
    using SM = CoopSmem<D, K>;
    constexpr int NREF = SM::NREF;
    static_assert(K % G == 0 && 32 % G == 0 && G >= 2, "group shape");
    extern __shared__ __align__(16) unsigned char coop_smem[];
    const int lane = threadIdx.x & 31, j = lane & (G - 1);
    const unsigned gm = group_mask<G>(lane);
    Real* ws = reinterpret_cast<Real*>(coop_smem) + (threadIdx.x / G) * SM::words;
    Real* sT = ws;
    Real* sQ = sT + SM::T;
    Real* sU = sQ + SM::Q;
    Real* sR = sU + SM::U;
    const int jl = (j + G - 1) % G, jr = (j + 1) % G;          // neighbour lanes (edges masked by hasL / hasR)
    const bool ring = sys0.ring != 0;
    const bool hasL = ring || j > 0, hasR = ring || j < NS - 1;

    for (;;) {
        unsigned long long base = 0;
        if (lane == 0) base = atomicAdd(a.counter, static_cast<unsigned long long>(32 / G));
        base = __shfl_sync(0xffffffffu, base, 0);
        if (base >= static_cast<unsigned long long>(a.n)) return;
        const i64 slot = static_cast<i64>(base) + lane / G;
        if (slot >= a.n) continue;
        const i64 i = a.order ? a.order[slot] : slot;

        const double Kc = a.Kp ? a.Kp[i] : sys0.K, eps = sys0.eps;   // per-orbit K (the one-thread kernel's sys.K)
        const i64 Ni = a.Np ? a.Np[i] : a.N;
        CoopSite<NS, Real, K> L;
        L.q = a.x_in[i * S + j];
        L.p = a.x_in[i * S + NS + j];
#pragma unroll
        for (int c = 0; c < K; ++c) {
            L.Wq[c] = static_cast<Real>(a.W_in[i * D * K + c * D + j]);
            L.Wp[c] = static_cast<Real>(a.W_in[i * D * K + c * D + NS + j]);
        }
        CoopQR<K, KPL> st;
#pragma unroll
        for (int m = 0; m < KPL; ++m) st.sums[m] = CS{0.0, 0.0};
        st.n = st.count_max = st.column = st.step = 0;
        st.G_max = st.orth_max = st.value = st.threshold = 0.0;
        st.code = 0;
        int8_t code = STATUS_OK;
        i64 hstep = 0, n = 0;
        bool alive = true, escaped = false;

        const i64 handoffs = Ni / a.tau;
        for (i64 h = 0; h < handoffs; ++h) {
            if (TAU_UNROLL > 1) {
#pragma unroll
                for (int t = 0; t < TAU_UNROLL; ++t) L.step(gm, jl, jr, hasL, hasR, Kc, eps);
            } else {
                for (int t = 0; t < a.tau; ++t) L.step(gm, jl, jr, hasL, hasR, Kc, eps);
            }
            n += a.tau;

            // ---- handoff: _status, then QRSpectrum(HouseholderQR) (orbit.jl:54-57) ----
            bool fw = true;
#pragma unroll
            for (int c = 0; c < K; ++c) fw = fw && isfin(L.Wq[c]) && isfin(L.Wp[c]);
            const bool fx = group_all<G>(gm, isfin(L.q) && isfin(L.p));
            fw = group_all<G>(gm, fw);
            int8_t c0 = fx ? (fw ? STATUS_OK : STATUS_W) : STATUS_STATE;
            if (c0 == STATUS_OK) {
                // stage the frame (column-major D x K; it stays there until the rows are reloaded)
#pragma unroll
                for (int c = 0; c < K; ++c) { sT[c * D + j] = L.Wq[c]; sT[c * D + NS + j] = L.Wp[c]; }
                __syncwarp(gm);
                Real A[KPL][D];   // this lane's columns: swept by the reflectors, then formed into Q in place
#pragma unroll
                for (int m = 0; m < KPL; ++m)
#pragma unroll
                    for (int r = 0; r < D; ++r) A[m][r] = sT[(j + m * G) * D + r];
                // _hh_sweep (householder.jl:19-50): reflector jj is built in place in shared memory by the owner of
                // column jj (zero when the column's norm is zero or not finite) and applied by every lane
                int count = 0;
#pragma unroll
                for (int jj = 0; jj < NREF; ++jj) {
                    const int owner = jj % G, mj = jj / G;
                    Real* u = sU + jj * D;
                    int okv = 0;
                    Real rho = Real(0);
                    if (j == owner) {
#pragma unroll
                        for (int m = 0; m < KPL; ++m)   // A[mj] with compile-time indices (jj need not unroll)
                            if (m == mj) {
#pragma unroll
                                for (int r = 0; r < D; ++r) u[r] = r >= jj ? A[m][r] : Real(0);
                            }
                        const Real cn = nrm<D>(u);
                        if (isfin(cn) && cn > Real(0)) {
                            const Real sg = u[jj] < Real(0) ? Real(-1) : Real(1);
                            u[jj] = u[jj] + sg * cn;
                            const Real nv = nrm<D>(u);
#pragma unroll
                            for (int r = 0; r < D; ++r) u[r] = dv(u[r], nv);
                            rho = -sg * cn;
                            okv = 1;
                        } else {
#pragma unroll
                            for (int r = 0; r < D; ++r) u[r] = Real(0);
                            rho = cn;
                        }
                    }
                    __syncwarp(gm);
                    if (__shfl_sync(gm, okv, owner, G)) {
#pragma unroll
                        for (int m = 0; m < KPL; ++m) {
                            const Real w = dotv<D>(u, A[m]);
#pragma unroll
                            for (int r = 0; r < D; ++r) A[m][r] = A[m][r] - (Real(2) * u[r]) * w;
                        }
                        count += 1;
                    }
                    if (j == owner) {
#pragma unroll
                        for (int m = 0; m < KPL; ++m)
#pragma unroll
                            for (int r = 0; r < D; ++r)
                                if (m == mj && r == jj) A[m][r] = rho;
                    }
                }
                // _finish (householder.jl:66-75): R's rows of this lane's columns, the signs of the diagonal (a bit
                // mask, read by every lane before any column is rewritten), then the sign-fixed upper triangle
#pragma unroll
                for (int m = 0; m < KPL; ++m)
#pragma unroll
                    for (int r = 0; r < K; ++r) sR[r + (j + m * G) * K] = A[m][r];
                __syncwarp(gm);
                unsigned neg = 0;
#pragma unroll
                for (int r = 0; r < K; ++r) neg |= (sR[r + r * K] < Real(0) ? 1u : 0u) << r;
                __syncwarp(gm);
#pragma unroll
                for (int m = 0; m < KPL; ++m) {
                    const int cc = j + m * G;
#pragma unroll
                    for (int r = 0; r < K; ++r) {
                        const Real sgr = (neg >> r) & 1u ? Real(-1) : Real(1);
                        sR[r + cc * K] = r > cc ? Real(0) : sgr * sR[r + cc * K];
                    }
                }
                // Q = the reflectors applied to I[:, 1:K] in reverse (householder.jl:77-80), then the signs
#pragma unroll
                for (int m = 0; m < KPL; ++m)
#pragma unroll
                    for (int r = 0; r < D; ++r) A[m][r] = r == j + m * G ? Real(1) : Real(0);
#pragma unroll
                for (int jj = NREF - 1; jj >= 0; --jj) {
                    const Real* u = sU + jj * D;
#pragma unroll
                    for (int m = 0; m < KPL; ++m) {
                        const Real w = dotv<D>(u, A[m]);
#pragma unroll
                        for (int r = 0; r < D; ++r) A[m][r] = A[m][r] - (Real(2) * u[r]) * w;
                    }
                }
#pragma unroll
                for (int m = 0; m < KPL; ++m) {
                    const int cc = j + m * G;
                    const Real sgc = (neg >> cc) & 1u ? Real(-1) : Real(1);
#pragma unroll
                    for (int r = 0; r < D; ++r) { A[m][r] = A[m][r] * sgc; sQ[cc * D + r] = A[m][r]; }
                }
                __syncwarp(gm);
                int status = QR_OK, fcol = 0;
#pragma unroll
                for (int jj = K - 1; jj >= 0; --jj) {
                    const Real pv = sR[jj + jj * K];
                    if (!(isfin(pv) && pv > Real(0))) { status = QR_PIVOT; fcol = jj + 1; }
                }
                // QRSpectrum's step (qr_spectrum.jl:36-74)
                bool replace = false;
                if (status != QR_OK) {
                    Real pv = sR[0];
#pragma unroll
                    for (int jj = 0; jj < K; ++jj) if (jj + 1 == fcol) pv = sR[jj + jj * K];
                    st.code = 1; st.column = fcol; st.value = static_cast<double>(pv);
                    st.threshold = isfin(pv) ? 0.0 : __longlong_as_double(0x7ff0000000000000LL);
                    st.step = n;
                } else {
                    const Real epsT = Eps<Real>::eps();
                    Real Gw = Real(0);
                    if (j == 0) Gw = window_Gw_sm<K>(sR, sU);   // the reflectors are spent: sU is scratch
                    Gw = __shfl_sync(gm, Gw, 0, G);
                    // orth_loss: this lane's columns of the upper triangle of Q'Q, then the maximum over the group
                    Real om = Real(0);
                    bool first = true;
#pragma unroll
                    for (int m = 0; m < KPL; ++m) {
                        const int cc = j + m * G;
#pragma unroll
                        for (int r = 0; r < K; ++r) {
                            if (r > cc) continue;
                            const Real* qi = sQ + r * D;
                            Real acc = qi[0] * A[m][0];
#pragma unroll
                            for (int l = 1; l < D; ++l) acc = fma(qi[l], A[m][l], acc);
                            if (r == cc) acc = acc - Real(1);
                            const Real av = fabs(acc);
                            om = first ? av : mx(om, av);
                            first = false;
                        }
                    }
#pragma unroll
                    for (int off = G / 2; off >= 1; off >>= 1) om = mx(om, __shfl_xor_sync(gm, om, off, G));
                    const Real orth = K >= 2 ? om : Real(0);
                    const Real thr = static_cast<Real>(a.prm[0].orthogonality_tol) * epsT * static_cast<Real>(K);
                    if (K >= 2 && !(orth <= thr)) {
                        st.code = 4; st.column = 0; st.value = static_cast<double>(orth);
                        st.threshold = static_cast<double>(thr); st.step = n;
                    } else {
#pragma unroll
                        for (int m = 0; m < KPL; ++m) cs_add(st.sums[m], lnr(sR[(j + m * G) * (K + 1)]));
                        const Real Gq = G_from_Gw<K>(Gw);
                        st.n = n;
                        st.G_max = jl_max(st.G_max, static_cast<double>(Gq));
                        st.orth_max = jl_max(st.orth_max, static_cast<double>(orth));
                        st.count_max = st.count_max > count ? st.count_max : count;
                        st.column = 0;
                        replace = true;
                    }
                }
                // W = Q (or the frame unchanged when the step failed)
                const Real* src = replace ? sQ : sT;
#pragma unroll
                for (int c = 0; c < K; ++c) { L.Wq[c] = src[c * D + j]; L.Wp[c] = src[c * D + NS + j]; }
                __syncwarp(gm);   // the workspace is free for the next handoff
                if (st.code != 0) c0 = STATUS_REDUCER;
            }
            if (c0 != STATUS_OK) { code = c0; hstep = n; alive = false; break; }
            if (a.escape > 0.0) {
                double mp = fabs(L.p);
#pragma unroll
                for (int off = G / 2; off >= 1; off >>= 1) mp = fmax(mp, __shfl_xor_sync(gm, mp, off, G));
                if (mp > a.escape) { escaped = true; break; }
            }
        }
        if (alive) {
            bool fw = true;
#pragma unroll
            for (int c = 0; c < K; ++c) fw = fw && isfin(L.Wq[c]) && isfin(L.Wp[c]);
            const bool fx = group_all<G>(gm, isfin(L.q) && isfin(L.p));
            const bool fin = fx && group_all<G>(gm, fw);
            code = escaped ? (fin ? STATUS_ESCAPED : (fx ? STATUS_W : STATUS_STATE))
                           : (n == Ni ? (fin ? STATUS_OK : (fx ? STATUS_W : STATUS_STATE)) : STATUS_OK);
            hstep = n;
        }
        a.x_out[i * S + j] = L.q;
        a.x_out[i * S + NS + j] = L.p;
#pragma unroll
        for (int c = 0; c < K; ++c) {
            a.W_out[i * D * K + c * D + j] = static_cast<double>(L.Wq[c]);
            a.W_out[i * D * K + c * D + NS + j] = static_cast<double>(L.Wp[c]);
        }
        // QRState<K> in the Julia layout: sums[K] (this lane's columns), then the scalars (lane 0 of the group)
        uint64_t* so = a.states + i * (sizeof(QRState<K>) / 8);
#pragma unroll
        for (int m = 0; m < KPL; ++m) {
            const int cc = j + m * G;
            so[2 * cc] = __double_as_longlong(st.sums[m].s);
            so[2 * cc + 1] = __double_as_longlong(st.sums[m].c);
        }
        if (j == 0) {
            QRState<K> full;
            uint64_t* fw_ = reinterpret_cast<uint64_t*>(&full);
#pragma unroll
            for (int w = 0; w < static_cast<int>(sizeof(QRState<K>) / 8); ++w) fw_[w] = 0;
            full.n = st.n; full.G_max = st.G_max; full.orth_max = st.orth_max; full.count_max = st.count_max;
            full.code = st.code; full.column = st.column; full.value = st.value; full.threshold = st.threshold;
            full.step = st.step;
#pragma unroll
            for (int w = 2 * K; w < static_cast<int>(sizeof(QRState<K>) / 8); ++w) so[w] = fw_[w];
            a.code[i] = code;
            if (a.hstep) a.hstep[i] = hstep;
        }
    }
}

template <int NS, typename Real, int K, int U, int MINB>
cudaError_t launch_coop_v(const cl_run& run, const EArgs& a, int grid, cudaStream_t st, LaunchInfo* info) {
    const SysChain<NS> sys = SysMaker<SysChain<NS>>::make(run, nullptr);
    auto k = coop_kernel<NS, Real, K, U, MINB>;
    const size_t smem = static_cast<size_t>(128 / NS) * CoopSmem<2 * NS, K>::words * sizeof(Real);
    // the workspace of one block can exceed the 48 KB default (d = 16 in Float64: 57 KB). The attribute belongs to
    // the current device's context, so it is set before every launch (a cheap, idempotent host call) rather than
    // cached once per process.
    const cudaError_t ea = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
    if (ea != cudaSuccess) return ea;
    k<<<grid, 128, smem, st>>>(a, sys);
    cudaError_t e = cudaGetLastError();
    if (info) {
        cudaFuncAttributes at;
        if (cudaFuncGetAttributes(&at, k) == cudaSuccess) info->regs = at.numRegs;
        info->block = 128;
        info->grid = grid;
    }
    return e;
}

template <int NS, typename Real, int K, int U>
cudaError_t launch_coop(const cl_run& run, const EArgs& a, int grid, const ETune& t, cudaStream_t st,
                        LaunchInfo* info) {
    const bool unrolled = U > 1 && t.unroll == U && a.tau == U;
    if (unrolled) {
        if (t.minb == 1) return launch_coop_v<NS, Real, K, U, 1>(run, a, grid, st, info);
        if (t.minb == 2) return launch_coop_v<NS, Real, K, U, 2>(run, a, grid, st, info);
        if (t.minb == 4) return launch_coop_v<NS, Real, K, U, 4>(run, a, grid, st, info);
    } else {
        if (t.minb == 1) return launch_coop_v<NS, Real, K, 1, 1>(run, a, grid, st, info);
        if (t.minb == 2) return launch_coop_v<NS, Real, K, 1, 2>(run, a, grid, st, info);
        if (t.minb == 4) return launch_coop_v<NS, Real, K, 1, 4>(run, a, grid, st, info);
    }
    return cudaErrorInvalidValue;
}

// Which ensemble instances have a cooperative form: lattices of NS = 2, 4 or 8 sites whose frame is reduced by
// QRSpectrum(HouseholderQR) alone, with k a multiple of NS.
template <class Sys, class F> struct CoopOf { static constexpr bool ok = false; static constexpr int NS = 0, K = 0; };
template <int NS_, int K_> struct CoopOf<SysChain<NS_>, Frame<K_, RQR<CL_QR_HOUSEHOLDER>>> {
    static constexpr int NS = NS_, K = K_;
    static constexpr bool ok = (NS == 2 || NS == 4 || NS == 8) && K % NS == 0;
};

// The ensemble launcher of the compiled menu: the cooperative kernel when the variant asks for NS lanes per orbit
// (and the class supplies W0: the cooperative kernel draws no seeded frames), else the one-thread kernel.
template <class Sys, typename Real, class F, int U>
cudaError_t launch_ensemble_any(const cl_run& run, const EArgs& a, int grid, const ETune& t, cudaStream_t st,
                                LaunchInfo* info) {
    if constexpr (CoopOf<Sys, F>::ok) {
        if (t.lanes > 1) {
            if (t.lanes != CoopOf<Sys, F>::NS || !a.W_in) return cudaErrorNotSupported;
            return launch_coop<CoopOf<Sys, F>::NS, Real, CoopOf<Sys, F>::K, U>(run, a, grid, t, st, info);
        }
    }
    return launch_ensemble<Sys, Real, F, U>(run, a, grid, t, st, info);
}

// Lanes per orbit of the cooperative form of a run (the lattice's site count), or 1 when it has none.
inline int coop_lanes(const cl_run& r) {
    if (r.sys.kind != CL_SYS_CHAIN || r.n_frames != 1) return 1;
    const cl_frame& f = r.frames[0];
    if (f.n_reducers != 1 || f.reducers[0].kind != CL_RED_QR || f.reducers[0].alg != CL_QR_HOUSEHOLDER) return 1;
    const int ns = r.d / 2;
    if ((ns != 2 && ns != 4 && ns != 8) || f.k % ns != 0) return 1;
    return ns;
}

}  // namespace cl
