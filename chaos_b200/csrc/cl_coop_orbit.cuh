// cl_coop_orbit.cuh -- `propagate`'s cooperative form for coupled standard-map lattices (StandardMapChain, d = 2 NS
// >= 8): one orbit per group of G lanes (G = 4 for NS = 4, 8 for NS = 5..8) instead of one per thread, so the d x k
// frame (128 entries at d = 16, k = 8, which spill in one thread) is spread over the group's registers and the
// orbit's steps over its lanes. It is the body of `_orbit_kernel!` / `_orbit_body` (src/Tangent/propagate.jl:32-50,
// orbit.jl:44-60) for one frame, with the launch window, carried state and frozen failed orbits of the one-thread
// kernel (cl_kernel.cuh).
//
// Between handoffs lane j < NS owns lattice site j: q_j, p_j (Float64) and rows j and NS + j of the frame; the step is
// CoopSite::step (cl_coop.cuh: the chain's tangent at the old point, ChainTangent * W with the neighbours' rows by
// warp shuffles, forward), the one-thread kernel's operations lane by lane. At a handoff the group checks the status
// (`_status`, orbit.jl:3) with a vote, stages the frame column-major in shared memory, and the frame's reducer chain
// runs on it there: QRSpectrum(HouseholderQR) column-parallel over the group (the reflectors built by the column
// owners in shared memory and applied by every lane to its own columns, as the ensemble's cooperative kernel does),
// QRSpectrum(MGS) and GALI in Float64 column-parallel by rounds (coop_qr_step, coop_gali_step), every other chain
// (in Float32 MGS and GALI, CGS / RGS / Givens QR, SALI, MEGNO, FLI, Benettin) by the group's first lane with the same
// reducer code as the one-thread kernel. Every entry is computed by the same operations in the same order and
// type, so the results are bit-identical to the one-thread kernel (and, in Float64, to the oracle).
#pragma once

#include "cl_coop.cuh"
#include "cl_registry.cuh"

namespace cl {

template <int NS> struct CoopWidth { static constexpr int G = NS <= 2 ? 2 : NS <= 4 ? 4 : 8; };

// QRSpectrum on the staged frame, column-parallel (qr_spectrum.jl:36-74): lane j owns columns j, j + G, ... The
// QRState sums of this lane's columns and the shared scalars (kept equal in every lane) are read from and written
// back to the Julia-layout state `st` in shared memory by lane 0 / the column owners. Returns true on failure.
//   HouseholderQR (householder.jl:19-80): the owner of column jj builds reflector jj in shared memory, every lane
//   applies it to its own columns and forms its own columns of Q.
//   MGS (orthonormalize.jl:49-58, 88-105): in round r the owner of column r, projected already on q_0 .. q_{r-1},
//   takes its norm and normalises it into q_r (the first column whose norm fails stops the factorisation, as the
//   serial loop does); then every lane projects its later columns on q_r (c = q_r . u, u - c q_r): each column sees
//   the same projections in the same order as in the serial loop.
template <int ALG, int D, int K, int G, typename Real>
__device__ __forceinline__ bool coop_qr_step(QRState<K>& st, i64 n, Real* sT, Real* sQ, Real* sU, Real* sR,
                                             unsigned gm, int j, double orth_tol) {
    constexpr int NREF = K < D ? K : K - 1;
    constexpr int KPL = (K + G - 1) / G;   // columns per lane (the last lanes may own fewer)
    constexpr bool HH = ALG == CL_QR_HOUSEHOLDER;
    Real A[KPL][D];
#pragma unroll
    for (int m = 0; m < KPL; ++m) {
        const int cc = j + m * G;
#pragma unroll
        for (int r = 0; r < D; ++r) A[m][r] = cc < K ? sT[cc * D + r] : Real(0);
    }
    int count = HH ? 0 : 1;
    int status = QR_OK, fcol = 0;
    if constexpr (!HH) {
        Real Rc[KPL][K];
#pragma unroll
        for (int m = 0; m < KPL; ++m)
#pragma unroll
            for (int i = 0; i < K; ++i) Rc[m][i] = Real(0);
#pragma unroll
        for (int rr = 0; rr < K; ++rr) {
            const int owner = rr % G, mo = rr / G;
            int bad = 0;
            if (j == owner) {
#pragma unroll
                for (int m = 0; m < KPL; ++m) {
                    if (m != mo) continue;
                    const Real gamma = nrm<D>(A[m]);
#pragma unroll
                    for (int i = 0; i < K; ++i) sR[i + rr * K] = i < rr ? Rc[m][i] : (i == rr ? gamma : Real(0));
                    if (!(isfin(gamma) && gamma > Real(0))) {
                        bad = 1;
                    } else {
#pragma unroll
                        for (int l = 0; l < D; ++l) { A[m][l] = dv(A[m][l], gamma); sQ[rr * D + l] = A[m][l]; }
                    }
                }
            }
            __syncwarp(gm);
            if (__shfl_sync(gm, bad, owner, G)) { status = QR_PIVOT; fcol = rr + 1; break; }
            const Real* qr_ = sQ + rr * D;
#pragma unroll
            for (int m = 0; m < KPL; ++m) {
                const int cc = j + m * G;
                if (cc <= rr || cc >= K) continue;
                const Real c = dotv<D>(qr_, A[m]);
                Rc[m][rr] = c;
#pragma unroll
                for (int l = 0; l < D; ++l) A[m][l] = A[m][l] - c * qr_[l];
            }
            __syncwarp(gm);
        }
    } else {
#pragma unroll
    for (int jj = 0; jj < NREF; ++jj) {
        const int owner = jj % G, mj = jj / G;
        Real* u = sU + jj * D;
        int okv = 0;
        Real rho = Real(0);
        if (j == owner) {
#pragma unroll
            for (int m = 0; m < KPL; ++m)
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
                if (j + m * G >= K) continue;
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
    // _finish (householder.jl:66-75)
#pragma unroll
    for (int m = 0; m < KPL; ++m) {
        const int cc = j + m * G;
        if (cc >= K) continue;
#pragma unroll
        for (int r = 0; r < K; ++r) sR[r + cc * K] = A[m][r];
    }
    __syncwarp(gm);
    unsigned neg = 0;
#pragma unroll
    for (int r = 0; r < K; ++r) neg |= (sR[r + r * K] < Real(0) ? 1u : 0u) << r;
    __syncwarp(gm);
#pragma unroll
    for (int m = 0; m < KPL; ++m) {
        const int cc = j + m * G;
        if (cc >= K) continue;
#pragma unroll
        for (int r = 0; r < K; ++r) {
            const Real sgr = (neg >> r) & 1u ? Real(-1) : Real(1);
            sR[r + cc * K] = r > cc ? Real(0) : sgr * sR[r + cc * K];
        }
    }
#pragma unroll
    for (int m = 0; m < KPL; ++m)
#pragma unroll
        for (int r = 0; r < D; ++r) A[m][r] = r == j + m * G ? Real(1) : Real(0);
#pragma unroll
    for (int jj = NREF - 1; jj >= 0; --jj) {
        const Real* u = sU + jj * D;
#pragma unroll
        for (int m = 0; m < KPL; ++m) {
            if (j + m * G >= K) continue;
            const Real w = dotv<D>(u, A[m]);
#pragma unroll
            for (int r = 0; r < D; ++r) A[m][r] = A[m][r] - (Real(2) * u[r]) * w;
        }
    }
#pragma unroll
    for (int m = 0; m < KPL; ++m) {
        const int cc = j + m * G;
        if (cc >= K) continue;
        const Real sgc = (neg >> cc) & 1u ? Real(-1) : Real(1);
#pragma unroll
        for (int r = 0; r < D; ++r) { A[m][r] = A[m][r] * sgc; sQ[cc * D + r] = A[m][r]; }
    }
    __syncwarp(gm);
#pragma unroll
    for (int jj = K - 1; jj >= 0; --jj) {
        const Real pv = sR[jj + jj * K];
        if (!(isfin(pv) && pv > Real(0))) { status = QR_PIVOT; fcol = jj + 1; }
    }
    }   // HouseholderQR
    bool replace = false, fail = false;
    if (status != QR_OK) {
        Real pv = sR[0];
#pragma unroll
        for (int jj = 0; jj < K; ++jj) if (jj + 1 == fcol) pv = sR[jj + jj * K];
        if (j == 0) {
            st.code = 1; st.column = fcol; st.value = static_cast<double>(pv);
            st.threshold = isfin(pv) ? 0.0 : __longlong_as_double(0x7ff0000000000000LL);
            st.step = n;
        }
        fail = true;
    } else {
        const Real epsT = Eps<Real>::eps();
        Real Gw = Real(0);
        if (j == 0) Gw = window_Gw_sm<K>(sR, sU);   // the reflectors are spent: sU is scratch
        Gw = __shfl_sync(gm, Gw, 0, G);
        // conditioning (the Gram-Schmidt family only, qr_spectrum.jl:54-58)
        if (!HH && !(static_cast<double>(Gw * epsT) < 0.5)) {
            if (j == 0) {
                st.code = 3; st.column = 0; st.value = static_cast<double>(Gw * epsT); st.threshold = 0.5; st.step = n;
            }
            __syncwarp(gm);
            return true;
        }
        Real om = Real(0);
        bool first = true;
#pragma unroll
        for (int m = 0; m < KPL; ++m) {
            const int cc = j + m * G;
            if (cc >= K) continue;
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
        // the maximum over the group: every lane owns at least one column (K >= G), and the NaN-aware maximum of
        // non-negative values does not depend on the order it combines them in
#pragma unroll
        for (int off = G / 2; off >= 1; off >>= 1) om = mx(om, __shfl_xor_sync(gm, om, off, G));
        const Real orth = K >= 2 ? om : Real(0);
        const Real thr = static_cast<Real>(orth_tol) * epsT * static_cast<Real>(K) * (HH ? Real(1) : Gw);
        if (K >= 2 && !(orth <= thr)) {
            if (j == 0) {
                st.code = 4; st.column = 0; st.value = static_cast<double>(orth);
                st.threshold = static_cast<double>(thr); st.step = n;
            }
            fail = true;
        } else {
#pragma unroll
            for (int m = 0; m < KPL; ++m) {
                const int cc = j + m * G;
                if (cc < K) cs_add(st.sums[cc], lnr(sR[cc * (K + 1)]));
            }
            if (j == 0) {
                const Real Gq = G_from_Gw<K>(Gw);
                st.n = n;
                st.G_max = jl_max(st.G_max, static_cast<double>(Gq));
                st.orth_max = jl_max(st.orth_max, static_cast<double>(orth));
                st.count_max = st.count_max > count ? st.count_max : count;
                st.column = 0;
            }
            replace = true;
        }
    }
    __syncwarp(gm);
    if (replace) {   // W = Q
#pragma unroll
        for (int m = 0; m < KPL; ++m) {
            const int cc = j + m * G;
            if (cc >= K) continue;
#pragma unroll
            for (int r = 0; r < D; ++r) sT[cc * D + r] = sQ[cc * D + r];
        }
    }
    __syncwarp(gm);
    return fail;
}

// GALI (gali.jl:17-201, the frame's unit columns and _gram_core! at :81-100) on the staged frame, column-parallel:
// every lane takes its own columns' norms, log sums and unit columns; the first failing column over the group (the
// lowest index) stops the step as the serial loop does. The twice-orthogonalised Gram core runs by rounds: in round r
// the owner of column r, projected already once on the final q_0 .. q_{r-1}, projects it a second time on all of them,
// takes its norm and normalises it, and G_r = G_{r-1} r_r is formed in every lane from the broadcast norm; then every
// lane makes the first projection of its later columns on q_r. Each column sees the serial loop's projections in its
// order. The frame becomes the unit columns (not Q). Returns true on failure.
template <int D, int K, int G, typename Real>
__device__ __forceinline__ bool coop_gali_step(GALIState<K>& st, i64 n, Real* sT, Real* sQ, unsigned gm, int j) {
    constexpr int KPL = (K + G - 1) / G;
    Real A[KPL][D], a[KPL];
    int mybad = K + 1;
#pragma unroll
    for (int m = KPL - 1; m >= 0; --m) {
        const int cc = j + m * G;
        if (cc >= K) continue;
#pragma unroll
        for (int r = 0; r < D; ++r) A[m][r] = sT[cc * D + r];
        a[m] = nrm<D>(A[m]);
        if (!(isfin(a[m]) && a[m] >= Eps<Real>::floatmin())) mybad = cc + 1;
    }
    const int bad = __reduce_min_sync(gm, static_cast<unsigned>(mybad));
    if (bad <= K) {
        const int owner = (bad - 1) % G, mo = (bad - 1) / G;
        Real v = Real(0);
#pragma unroll
        for (int m = 0; m < KPL; ++m) if (m == mo) v = a[m];
        v = __shfl_sync(gm, v, owner, G);
        if (j == 0) { st.value = static_cast<double>(v); st.step = n; st.code = 1; st.column = bad; }
        __syncwarp(gm);
        return true;
    }
#pragma unroll
    for (int m = 0; m < KPL; ++m) {
        const int cc = j + m * G;
        if (cc >= K) continue;
        CS acc{st.s[cc], st.c[cc]};
        cs_add(acc, lnr(a[m]));
        st.s[cc] = acc.s; st.c[cc] = acc.c;
#pragma unroll
        for (int r = 0; r < D; ++r) { A[m][r] = dv(A[m][r], a[m]); sT[cc * D + r] = A[m][r]; }
    }
    Real g = Real(1);
#pragma unroll
    for (int rr = 0; rr < K; ++rr) {
        const int owner = rr % G, mo = rr / G;
        Real rn = Real(0);
        if (j == owner) {
#pragma unroll
            for (int m = 0; m < KPL; ++m) {
                if (m != mo) continue;
#pragma unroll
                for (int p = 0; p < rr; ++p) {   // the second pass
                    const Real* qp = sQ + p * D;
                    Real cc = Real(0);
#pragma unroll
                    for (int i = 0; i < D; ++i) cc = cc + qp[i] * A[m][i];
#pragma unroll
                    for (int i = 0; i < D; ++i) A[m][i] = A[m][i] - cc * qp[i];
                }
                rn = nrm<D>(A[m]);
                const Real sc = rn == Real(0) ? Real(1) : rn;
#pragma unroll
                for (int i = 0; i < D; ++i) { A[m][i] = dv(A[m][i], sc); sQ[rr * D + i] = A[m][i]; }
            }
        }
        rn = __shfl_sync(gm, rn, owner, G);
        if (rr > 0) {
            g = g * rn;
            if (j == owner) st.gali[rr - 1] = static_cast<double>(g);
        }
        __syncwarp(gm);
        const Real* qr_ = sQ + rr * D;
#pragma unroll
        for (int m = 0; m < KPL; ++m) {   // the first pass of the later columns on q_rr
            const int cc = j + m * G;
            if (cc <= rr || cc >= K) continue;
            Real c = Real(0);
#pragma unroll
            for (int i = 0; i < D; ++i) c = c + qr_[i] * A[m][i];
#pragma unroll
            for (int i = 0; i < D; ++i) A[m][i] = A[m][i] - c * qr_[i];
        }
    }
    if (j == 0) st.n = n;
    __syncwarp(gm);
    return false;
}

// The column-parallel QR runs when every lane owns at least one column (K >= G): HouseholderQR in both precisions,
// MGS in Float64 (in Float32 its rounds ran slower than the first lane's serial MGS: d = 16, 2048 orbits, 36.8
// against 22.5 ms; in Float64 116 against 119 ms, 8192 orbits 246 against 280 ms); other chains on the first lane.
template <class F, typename Real, int G> struct CoopQRForm { static constexpr bool value = false; static constexpr int alg = 0; };
template <int KK, int ALG, typename Real, int G> struct CoopQRForm<Frame<KK, RQR<ALG>>, Real, G> {
    static constexpr bool value = KK >= G && (ALG == CL_QR_HOUSEHOLDER || (ALG == CL_QR_MGS && sizeof(Real) == 8));
    static constexpr int alg = ALG;
};

// GALI (without SALI) runs column-parallel in Float64 when every lane owns at least one column.
template <class F, typename Real, int G> struct CoopGaliForm { static constexpr bool value = false; };
template <int KK, typename Real, int G> struct CoopGaliForm<Frame<KK, RGALI<false>>, Real, G> {
    static constexpr bool value = KK >= G && KK >= 2 && sizeof(Real) == 8;
};

template <int NS, typename Real, class F0>
__global__ void __launch_bounds__(128) coop_orbit_kernel(const KArgs a, const SysChain<NS> sys) {
    constexpr int G = CoopWidth<NS>::G, D = 2 * NS, S = 2 * NS, K = F0::K;
    using Ch = typename F0::template Chain_<D>;
    constexpr int words = Ch::bytes / 8;
    constexpr bool HH = CoopQRForm<F0, Real, G>::value || CoopGaliForm<F0, Real, G>::value;   // shared-memory workspace
    constexpr int NREF = K < D ? K : K - 1;
    // per group: the staged frame, then (Householder) Q, the reflectors and R, then the chain's state
    constexpr int FW = D * K, QW = HH ? D * K : 0, UW = HH ? (D * NREF > K ? D * NREF : K) : 0, RW = HH ? K * K : 0;
    constexpr int REAL_WORDS = FW + QW + UW + RW;
    constexpr int GROUP_BYTES = ((REAL_WORDS * static_cast<int>(sizeof(Real)) + 7) / 8) * 8 + words * 8;
    static_assert(32 % G == 0 && G >= NS, "group shape");
    extern __shared__ __align__(16) unsigned char coop_orbit_smem[];
    const int lane = threadIdx.x & 31, j = lane & (G - 1);
    const unsigned gm = group_mask<G>(lane);
    const i64 i = (static_cast<i64>(blockIdx.x) * blockDim.x + threadIdx.x) / G;
    if (i >= a.n) return;   // whole groups: G divides the block
    unsigned char* gbase = coop_orbit_smem + (threadIdx.x / G) * GROUP_BYTES;
    Real* sT = reinterpret_cast<Real*>(gbase);
    Real* sQ = sT + FW;
    Real* sU = sQ + QW;
    Real* sR = sU + UW;
    uint64_t* sSt = reinterpret_cast<uint64_t*>(gbase + ((REAL_WORDS * static_cast<int>(sizeof(Real)) + 7) / 8) * 8);
    const bool site = j < NS;
    const int jl = (j + NS - 1) % NS, jr = (j + 1) % NS;
    const bool ring = sys.ring != 0;
    const bool hasL = site && (ring || j > 0), hasR = site && (ring || j < NS - 1);
    const bool fresh = a.n0 == 0;
    const i64 xso = a.soa ? 1 : S, xsc = a.soa ? a.n : 1;
    const i64 wso = a.soa ? 1 : D * K, wsc = a.soa ? a.n : 1;

    CoopSite<NS, Real, K, G> L;
    L.q = site ? a.x_in[i * xso + j * xsc] : 0.0;
    L.p = site ? a.x_in[i * xso + (NS + j) * xsc] : 0.0;
    int8_t code = STATUS_OK;
    i64 hstep = 0;
    if (fresh && !a.W_in[0]) {
        if (j == 0) seeded_frame<D, K>(a.seed, a.orbit_base + i + 1, sT);
        __syncwarp(gm);
#pragma unroll
        for (int c = 0; c < K; ++c) {
            L.Wq[c] = site ? sT[c * D + j] : Real(0);
            L.Wp[c] = site ? sT[c * D + NS + j] : Real(0);
        }
        __syncwarp(gm);
    } else {
#pragma unroll
        for (int c = 0; c < K; ++c) {
            L.Wq[c] = site ? static_cast<Real>(a.W_in[0][i * wso + (c * D + j) * wsc]) : Real(0);
            L.Wp[c] = site ? static_cast<Real>(a.W_in[0][i * wso + (c * D + NS + j) * wsc]) : Real(0);
        }
    }
    // the chain's state lives in shared memory (Julia layout), loaded or zeroed by the group's lanes
    if (fresh) {
        for (int w = j; w < words; w += G) sSt[w] = 0;
    } else {
        for (int w = j; w < words; w += G) sSt[w] = a.states[0][i * words + w];
        code = a.code[0][i];
        hstep = a.hstep[0] ? a.hstep[0][i] : 0;
    }
    if (code != STATUS_OK) return;   // frozen since an earlier launch: nothing is rewritten
    __syncwarp(gm);

    i64 n = a.n0;
    bool alive = true;
    const i64 handoffs = a.steps / a.tau;
    for (i64 h = 0; h < handoffs; ++h) {
        for (int t = 0; t < a.tau; ++t) L.step(gm, jl, jr, hasL, hasR, sys.K, sys.eps);
        n += a.tau;
        // _status, then the chain, then _any_failed (orbit.jl:54-57)
        bool fw = true;
#pragma unroll
        for (int c = 0; c < K; ++c) fw = fw && isfin(L.Wq[c]) && isfin(L.Wp[c]);
        const bool fx = group_all<G>(gm, !site || (isfin(L.q) && isfin(L.p)));
        fw = group_all<G>(gm, !site || fw);
        int8_t c0 = fx ? (fw ? STATUS_OK : STATUS_W) : STATUS_STATE;
        if (c0 == STATUS_OK) {
            if (site) {
#pragma unroll
                for (int c = 0; c < K; ++c) { sT[c * D + j] = L.Wq[c]; sT[c * D + NS + j] = L.Wp[c]; }
            }
            __syncwarp(gm);
            int failed = 0;
            if constexpr (CoopQRForm<F0, Real, G>::value) {
                QRState<K>& st = *reinterpret_cast<QRState<K>*>(sSt);
                failed = coop_qr_step<CoopQRForm<F0, Real, G>::alg, D, K, G>(st, n, sT, sQ, sU, sR, gm, j, a.prm[0][0].orthogonality_tol) ? 1 : 0;
            } else if constexpr (CoopGaliForm<F0, Real, G>::value) {
                GALIState<K>& st = *reinterpret_cast<GALIState<K>*>(sSt);
                failed = coop_gali_step<D, K, G>(st, n, sT, sQ, gm, j) ? 1 : 0;
            } else {
                if (j == 0) {
                    Ch ch;
                    ch.load(sSt);
                    ch.step(n, sT, a.prm[0]);
                    failed = ch.failed() ? 1 : 0;
                    ch.store(sSt);
                }
                failed = __shfl_sync(gm, failed, 0, G);
                __syncwarp(gm);
            }
            if (site) {
#pragma unroll
                for (int c = 0; c < K; ++c) { L.Wq[c] = sT[c * D + j]; L.Wp[c] = sT[c * D + NS + j]; }
            }
            __syncwarp(gm);
            if (failed) c0 = STATUS_REDUCER;
        }
        if (c0 != STATUS_OK) { code = c0; hstep = n; alive = false; break; }
    }
    if (alive) {   // orbit.jl:58: the final status check runs only at step N
        bool fw = true;
#pragma unroll
        for (int c = 0; c < K; ++c) fw = fw && isfin(L.Wq[c]) && isfin(L.Wp[c]);
        const bool fx = group_all<G>(gm, !site || (isfin(L.q) && isfin(L.p)));
        fw = group_all<G>(gm, !site || fw);
        code = n == a.N ? (fx ? (fw ? STATUS_OK : STATUS_W) : STATUS_STATE) : STATUS_OK;
        hstep = n;
    }
    if (site) {
        a.x_out[i * xso + j * xsc] = L.q;
        a.x_out[i * xso + (NS + j) * xsc] = L.p;
#pragma unroll
        for (int c = 0; c < K; ++c) {
            a.W_out[0][i * wso + (c * D + j) * wsc] = static_cast<double>(L.Wq[c]);
            a.W_out[0][i * wso + (c * D + NS + j) * wsc] = static_cast<double>(L.Wp[c]);
        }
    }
    __syncwarp(gm);
    for (int w = j; w < words; w += G) a.states[0][i * words + w] = sSt[w];
    if (j == 0) {
        a.code[0][i] = code;
        if (a.hstep[0]) a.hstep[0][i] = hstep;
    }
}

template <int NS, typename Real, class F0>
cudaError_t launch_coop_orbit(const cl_run& run, const KArgs& a, cudaStream_t st, LaunchInfo* info) {
    constexpr int G = CoopWidth<NS>::G, D = 2 * NS, K = F0::K;
    constexpr bool HH = CoopQRForm<F0, Real, G>::value || CoopGaliForm<F0, Real, G>::value;   // shared-memory workspace
    constexpr int NREF = K < D ? K : K - 1;
    constexpr int FW = D * K, QW = HH ? D * K : 0, UW = HH ? (D * NREF > K ? D * NREF : K) : 0, RW = HH ? K * K : 0;
    constexpr int words = F0::template Chain_<D>::bytes / 8;
    constexpr int GROUP_BYTES = (((FW + QW + UW + RW) * static_cast<int>(sizeof(Real)) + 7) / 8) * 8 + words * 8;
    const SysChain<NS> sys = SysMaker<SysChain<NS>>::make(run, nullptr);
    auto k = coop_orbit_kernel<NS, Real, F0>;
    const int block = 128;
    const int smem = (block / G) * GROUP_BYTES;
    if (smem > 48 * 1024) {
        const cudaError_t ea = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
        if (ea != cudaSuccess) return ea;
    }
    const long long grid = (a.n * G + block - 1) / block;
    k<<<static_cast<unsigned>(grid), block, smem, st>>>(a, sys);
    const cudaError_t e = cudaGetLastError();
    if (info) {
        cudaFuncAttributes at;
        if (cudaFuncGetAttributes(&at, k) == cudaSuccess) info->regs = at.numRegs;
        info->block = block;
        info->grid = static_cast<int>(grid);
    }
    return e;
}

// The variant number of the cooperative form in a lattice instance's variant set (bit V_COOP - 1 of its mask).
constexpr int V_COOP = 8;

// Orbits up to which an untuned run takes the cooperative form. Measured at N = 2e4, tau = 10, k = 8 (ms, one-thread
// / cooperative): d = 16 at 512 and 2048 orbits 1.6-3x faster cooperatively (Float64 MGS 232 / 116, Float64 GALI
// 295 / 186, mixed Householder 120 / 41), at 8192 about even (Float64 Householder 329 / 304, Float64 GALI 303 / 401),
// slower at 65536 orbits (Float64 Householder 127 / 213 at N = 2000), where one thread per orbit already fills the
// GPU; d = 8 Float64 1.2-1.9x faster at 2048 and 8192 (GALI 135 / 71).
constexpr i64 kCoopMaxOrbits = 4096;

// A lattice instance of `propagate` with d >= 8: variant 1 is the one-thread kernel, variant V_COOP the cooperative
// form; an untuned run (any other variant number) takes the cooperative form for ensembles of at most
// kCoopMaxOrbits orbits, where one thread per orbit leaves most of the GPU idle. The tuner times both on long runs.
template <int NS, typename Real, class F0>
cudaError_t launch_chain_instance(const cl_run& run, const KArgs& a, const double* devA, cudaStream_t st,
                                  LaunchInfo* info, int minb) {
    const bool coop = minb == V_COOP || (minb != 1 && a.n <= kCoopMaxOrbits);
    if (!coop) return launch_variant<SysChain<NS>, Real, F0, Frame<1>, Frame<1>, 1, 1>(run, a, devA, st, info);
    return launch_coop_orbit<NS, Real, F0>(run, a, st, info);
}

}  // namespace cl
