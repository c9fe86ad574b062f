// cl_reducers.cuh -- the reducers fused into the orbit kernel: QRSpectrum (all six orthonormalisers), Benettin,
// SALI, GALI, MEGNO and FLI, and RLI for the pair streams of the indicator recorder. Each is a tag type with
//   State<D, K>                the isbits layout of the reference's state struct with T = Float64
//   step(st, n, W, prm)        `reducer_step` (src/Tangent/Tangent.jl:44-49): never throws, records failures
//   failed(st)                 `reducer_failed`
// and its own `replace` semantics on the frame W (d x K, column-major, registers). With Real = double every
// operation is the reference's, in its order; with Real = float (mixed kernels) the frame, norms and QR are
// Float32 while the logarithms and their Neumaier sums stay Float64.
#pragma once

#include "cl_math.cuh"
#include "cl_qr.cuh"

namespace cl {

typedef int64_t i64;

struct RedParams { double orthogonality_tol; };

// ---- QRSpectrum (src/Lyapunov/qr_spectrum.jl:14-96) -------------------------------------------------------------------
template <int K> struct QRState {
    CS sums[K]; i64 n; double G_max, orth_max; i64 count_max; int8_t code; i64 column; double value, threshold; i64 step;
};
static_assert(sizeof(QRState<2>) == 16 * 2 + 72 && sizeof(QRState<8>) == 16 * 8 + 72, "QRState layout");

template <int ALG>
struct RQR {
    static constexpr int kind = CL_RED_QR;
    template <int D, int K> using State = QRState<K>;
    template <int D, int K, typename T>
    static __device__ __forceinline__ void step(State<D, K>& st, i64 n, T* W, const RedParams& prm) {
        if (st.code != 0) return;
        T Q[D * K], R[K * K];
        const QRRes f = orthonormalize<ALG, D, K>(W, Q, R);
        if (f.status != QR_OK) {   // _factor_failure, qr_spectrum.jl:43-48
            if (f.status == QR_PASSES) {
                st.code = 2; st.column = f.column; st.value = MAX_PASSES + 1; st.threshold = MAX_PASSES;
            } else {
                T pv = R[0];
#pragma unroll
                for (int j = 0; j < K; ++j) if (j + 1 == f.column) pv = R[j + j * K];
                st.code = 1; st.column = f.column; st.value = static_cast<double>(pv);
                st.threshold = isfin(pv) ? 0.0 : __longlong_as_double(0x7ff0000000000000LL);
            }
            st.step = n;
            return;
        }
        const T eps = Eps<T>::eps();
        const T Gw = window_Gw<K>(R);
        constexpr bool gs = ALG == CL_QR_CGS || ALG == CL_QR_MGS || ALG == CL_QR_RGS;
        if (gs && !(static_cast<double>(Gw * eps) < 0.5)) {   // conditioning (GS family only)
            st.code = 3; st.column = 0; st.value = static_cast<double>(Gw * eps); st.threshold = 0.5; st.step = n;
            return;
        }
        const T orth = K >= 2 ? orth_loss<D, K>(Q) : T(0);
        const T g = (ALG == CL_QR_CGS || ALG == CL_QR_MGS) ? Gw : T(1);
        const T thr = static_cast<T>(prm.orthogonality_tol) * eps * static_cast<T>(K) * g;
        if (K >= 2 && !(orth <= thr)) {
            st.code = 4; st.column = 0; st.value = static_cast<double>(orth); st.threshold = static_cast<double>(thr);
            st.step = n;
            return;
        }
#pragma unroll
        for (int i = 0; i < K; ++i) cs_add(st.sums[i], lnr(R[i + i * K]));
        const T G = G_from_Gw<K>(Gw);
        st.n = n;
        st.G_max = jl_max(st.G_max, static_cast<double>(G));
        st.orth_max = jl_max(st.orth_max, static_cast<double>(orth));
        st.count_max = st.count_max > f.count ? st.count_max : f.count;
        st.column = 0;
#pragma unroll
        for (int l = 0; l < D * K; ++l) W[l] = Q[l];
    }
    template <int D, int K>
    static __device__ __forceinline__ bool failed(const State<D, K>& st) { return st.code != 0; }
};

// ---- Benettin (src/Lyapunov/benettin.jl:11-53) --------------------------------------------------------------------
struct BenettinState { CS sum; i64 n; int8_t code; double value; i64 step; };
static_assert(sizeof(BenettinState) == 48, "BenettinState layout");

struct RBenettin {
    static constexpr int kind = CL_RED_BENETTIN;
    template <int D, int K> using State = BenettinState;
    template <int D, int K, typename T>
    static __device__ __forceinline__ void step(State<D, K>& st, i64 n, T* W, const RedParams&) {
        if (st.code != 0) return;
        const T alpha = nrm<D>(W);
        if (!(isfin(alpha) && alpha > T(0))) { st.code = 1; st.value = static_cast<double>(alpha); st.step = n; return; }
        cs_add(st.sum, lnr(alpha));
        st.n = n;
#pragma unroll
        for (int l = 0; l < D * K; ++l) W[l] = dv(W[l], alpha);
    }
    template <int D, int K>
    static __device__ __forceinline__ bool failed(const State<D, K>& st) { return st.code != 0; }
};

// ---- SALI (src/Indicators/sali.jl:14-68) ---------------------------------------------------------------------------
struct SALIState { CS s1, s2; double sali, value; i64 n, step; int8_t code, column; };
static_assert(sizeof(SALIState) == 72, "SALIState layout");

// Column-norm failure record shared by SALI, MEGNO and FLI (sali.jl:102-106): column 1 unless only column 2 fails.
template <typename St, typename T>
__device__ __forceinline__ bool pair_norms(St& st, i64 n, T a1, T a2) {
    const bool ok1 = isfin(a1) && a1 > T(0), ok2 = isfin(a2) && a2 > T(0);
    if (ok1 && ok2) return true;
    st.column = ok1 ? 2 : 1; st.value = static_cast<double>(ok1 ? a2 : a1); st.step = n; st.code = 1;
    return false;
}

struct RSALI {
    static constexpr int kind = CL_RED_SALI;
    template <int D, int K> using State = SALIState;
    template <int D, int K, typename T>
    static __device__ __forceinline__ void step(State<D, K>& st, i64 n, T* W, const RedParams&) {
        if (st.code != 0) return;
        const T a1 = nrm<D>(W), a2 = nrm<D>(W + D);
        if (!pair_norms(st, n, a1, a2)) return;
        T dm[D], dp[D];
#pragma unroll
        for (int i = 0; i < D; ++i) {
            const T u1 = dv(W[i], a1), u2 = dv(W[D + i], a2);
            W[i] = u1; W[D + i] = u2;
            dm[i] = u1 - u2; dp[i] = u1 + u2;
        }
        cs_add(st.s1, lnr(a1));
        cs_add(st.s2, lnr(a2));
        st.sali = static_cast<double>(jl_min(nrm<D>(dm), nrm<D>(dp)));
        st.n = n;
    }
    template <int D, int K>
    static __device__ __forceinline__ bool failed(const State<D, K>& st) { return st.code != 0; }
};

// ---- GALI (src/Indicators/gali.jl:17-201) --------------------------------------------------------------------------
template <int K> struct GALIState { double s[K], c[K], gali[K - 1]; double value; i64 n, step; int8_t code; i64 column; };
static_assert(sizeof(GALIState<4>) == 24 * 4 + 32, "GALIState layout");

template <int K, bool WITH_SALI> struct GALIFrameState { GALIState<K> g; };
template <int K> struct GALIFrameState<K, true> { GALIState<K> g; SALIState s; };

// GALI; with WITH_SALI also the SALI of the frame's first two columns. A separate SALI run (k = 2) on the same orbit
// and W0 is bitwise GALI's columns 1-2 (test/gali/ga_ac05_08.jl:356-397): same norms, same Neumaier sums, same unit
// columns. So the chain (GALI, SALI) of one frame gives both records, laid out as the tuple (GALIState, SALIState);
// the SALI record stops with the frame when GALI fails on a column SALI does not read.
template <bool WITH_SALI>
struct RGALI {
    static constexpr int kind = CL_RED_GALI;
    template <int D, int K> using State = GALIFrameState<K, WITH_SALI>;
    template <int D, int K, typename T>
    static __device__ __forceinline__ void step(State<D, K>& S, i64 n, T* W, const RedParams&) {
        GALIState<K>& st = S.g;
        if (st.code != 0) return;
        T a[K];
#pragma unroll
        for (int j = 0; j < K; ++j) a[j] = nrm<D>(W + j * D);   // _norm_col
        bool sali_ok = true;
        if constexpr (WITH_SALI) sali_ok = S.s.code == 0 && pair_norms(S.s, n, a[0], a[1]);
        int bad = 0;
#pragma unroll
        for (int j = K - 1; j >= 0; --j)
            if (!(isfin(a[j]) && a[j] >= Eps<T>::floatmin())) bad = j + 1;
        if (bad != 0) {
            T v = a[0];
#pragma unroll
            for (int j = 0; j < K; ++j) if (j + 1 == bad) v = a[j];
            st.value = static_cast<double>(v); st.step = n; st.code = 1; st.column = bad;
            return;
        }
#pragma unroll
        for (int j = 0; j < K; ++j) {
            CS acc{st.s[j], st.c[j]};
            cs_add(acc, lnr(a[j]));
            st.s[j] = acc.s; st.c[j] = acc.c;
        }
        T Q[D * K];
#pragma unroll
        for (int j = 0; j < K; ++j)
#pragma unroll
            for (int i = 0; i < D; ++i) { const T u = dv(W[i + j * D], a[j]); W[i + j * D] = u; Q[i + j * D] = u; }
        if constexpr (WITH_SALI) {
            if (sali_ok) {   // sali.jl:107-110 on the unit columns 1-2
                T dm[D], dp[D];
#pragma unroll
                for (int i = 0; i < D; ++i) { dm[i] = W[i] - W[D + i]; dp[i] = W[i] + W[D + i]; }
                S.s.s1 = CS{st.s[0], st.c[0]};
                S.s.s2 = CS{st.s[1], st.c[1]};
                S.s.sali = static_cast<double>(jl_min(nrm<D>(dm), nrm<D>(dp)));
                S.s.n = n;
            }
        }
        T g = T(1);   // _gram_core!, gali.jl:81-100
#pragma unroll
        for (int j = 0; j < K; ++j) {
#pragma unroll
            for (int pass = 0; pass < 2; ++pass)
#pragma unroll
                for (int p = 0; p < j; ++p) {
                    T cc = T(0);
#pragma unroll
                    for (int i = 0; i < D; ++i) cc = cc + Q[i + p * D] * Q[i + j * D];
#pragma unroll
                    for (int i = 0; i < D; ++i) Q[i + j * D] = Q[i + j * D] - cc * Q[i + p * D];
                }
            const T r = nrm<D>(Q + j * D);
            const T sc = r == T(0) ? T(1) : r;
#pragma unroll
            for (int i = 0; i < D; ++i) Q[i + j * D] = dv(Q[i + j * D], sc);
            if (j > 0) { g = g * r; st.gali[j - 1] = static_cast<double>(g); }
        }
        st.n = n;
    }
    template <int D, int K>
    static __device__ __forceinline__ bool failed(const State<D, K>& S) {
        if constexpr (WITH_SALI) return S.g.code != 0 || S.s.code != 0;
        return S.g.code != 0;
    }
};

// ---- MEGNO (src/Indicators/megno.jl:29-113) -------------------------------------------------------------------------
struct MegnoSums { CS s, R1, R2, Q, Q2; };
struct MEGNOState { MegnoSums c1, c2; double value; i64 n, K, step; int8_t code, column; };
static_assert(sizeof(MEGNOState) == 200, "MEGNOState layout");

__device__ __forceinline__ void megno_add(MegnoSums& m, double a, i64 n) {   // megno.jl:63-67
    const double tn = static_cast<double>(n);
    cs_add(m.R1, tn * a);
    cs_add(m.R2, tn * tn * a);
    cs_add(m.s, a);
    cs_add(m.Q, 2 * cs_total(m.R1) / tn);
    cs_add(m.Q2, 3 * cs_total(m.R2));
}

template <bool REPLACE>
struct RMEGNO {
    static constexpr int kind = CL_RED_MEGNO;
    template <int D, int K> using State = MEGNOState;
    template <int D, int K, typename T>
    static __device__ __forceinline__ void step(State<D, K>& st, i64 n, T* W, const RedParams&) {
        if (st.code != 0) return;
        const T a1 = nrm<D>(W), a2 = nrm<D>(W + D);
        if (!pair_norms(st, n, a1, a2)) return;
        megno_add(st.c1, lnr(a1), n);
        megno_add(st.c2, lnr(a2), n);
        st.n = n; st.K = st.K + 1;
        if (REPLACE) {
#pragma unroll
            for (int i = 0; i < D; ++i) { W[i] = dv(W[i], a1); W[D + i] = dv(W[D + i], a2); }
        }
    }
    template <int D, int K>
    static __device__ __forceinline__ bool failed(const State<D, K>& st) { return st.code != 0; }
};

// ---- FLI (src/Indicators/fli.jl:26-96) -------------------------------------------------------------------------------
struct FLIState { CS s1, s2; double f1, fB, value; i64 n, step, step1, stepB; int8_t code, column, colB; };
static_assert(sizeof(FLIState) == 96, "FLIState layout");

template <bool REPLACE>
struct RFLI {
    static constexpr int kind = CL_RED_FLI;
    template <int D, int K> using State = FLIState;
    template <int D, int K, typename T>
    static __device__ __forceinline__ void step(State<D, K>& st, i64 n, T* W, const RedParams&) {
        if (st.code != 0) return;
        const T a1 = nrm<D>(W), a2 = nrm<D>(W + D);
        if (!pair_norms(st, n, a1, a2)) return;
        cs_add(st.s1, lnr(a1));
        cs_add(st.s2, lnr(a2));
        const double S1 = cs_total(st.s1), S2 = cs_total(st.s2);   // fli_maxima, fli.jl:54-60
        if (S1 > st.f1) { st.f1 = S1; st.step1 = n; }
        if (S1 > st.fB) { st.fB = S1; st.stepB = n; st.colB = 1; }
        if (S2 > st.fB) { st.fB = S2; st.stepB = n; st.colB = 2; }
        st.n = n;
        if (REPLACE) {
#pragma unroll
            for (int i = 0; i < D; ++i) { W[i] = dv(W[i], a1); W[D + i] = dv(W[D + i], a2); }
        }
    }
    template <int D, int K>
    static __device__ __forceinline__ bool failed(const State<D, K>& st) { return st.code != 0; }
};

// ---- RLI (src/Indicators/rli.jl:24-114) -------------------------------------------------------------------------
// On a pair stream (PairMap, d = 2h): the two arriving columns, (xi; 0) of orbit A and (0; xi) of orbit B, Benettin's
// log sums per column, DL = |S_B - S_A| / n with the correction terms split out, and the compensated sum Q of the DL
// series; the off-block entries must stay exactly 0 (code 2, "pairing").
struct RLIState { CS sA, sB, Q; double value; i64 n, K, step; int8_t code, column; };
static_assert(sizeof(RLIState) == 88, "RLIState layout");

template <bool REPLACE>
struct RRLI {
    static constexpr int kind = CL_RED_RLI;
    template <int D, int K> using State = RLIState;
    template <int D, int K, typename T>
    static __device__ __forceinline__ void step(State<D, K>& st, i64 n, T* W, const RedParams&) {
        if (st.code != 0) return;
        const T a1 = nrm<D>(W), a2 = nrm<D>(W + D);
        if (!pair_norms(st, n, a1, a2)) return;
        constexpr int h = D / 2;
        T m1 = T(0), m2 = T(0);   // _offblock, rli.jl:58-65
#pragma unroll
        for (int i = 0; i < h; ++i) { m1 = jl_max(m1, fabs(W[h + i])); m2 = jl_max(m2, fabs(W[D + i])); }
        if (!(m1 == T(0) && m2 == T(0))) {
            const bool first_clean = m1 == T(0);
            st.column = first_clean ? 2 : 1; st.value = static_cast<double>(first_clean ? m2 : m1); st.step = n; st.code = 2;
            return;
        }
        cs_add(st.sA, lnr(a1));
        cs_add(st.sB, lnr(a2));
        cs_add(st.Q, fabs((st.sB.s - st.sA.s) + (st.sB.c - st.sA.c)) / static_cast<double>(n));   // rli_dl, rli.jl:53
        st.n = n;
        st.K = st.K + 1;
        if (REPLACE) {
#pragma unroll
            for (int i = 0; i < D; ++i) { W[i] = dv(W[i], a1); W[D + i] = dv(W[D + i], a2); }
        }
    }
    template <int D, int K>
    static __device__ __forceinline__ bool failed(const State<D, K>& st) { return st.code != 0; }
};

}  // namespace cl
