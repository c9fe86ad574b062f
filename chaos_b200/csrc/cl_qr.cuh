// cl_qr.cuh -- the QR family of QRSpectrum in registers: Gram-Schmidt (CGS / MGS / RGS), Householder, augmented
// Householder and Givens, window_Gw, orth_loss. Templated on the tangent dimension D, the number of deviation
// vectors K and the element type (double for the plain kernel, float for the mixed one); every loop bound is a
// template constant, so the matrices stay in registers.
//
// Operation order follows the reference exactly (src/Lyapunov/orthonormalize.jl, householder.jl, qr_spectrum.jl):
// dot products and sums are left folds of plain products (StaticArrays `_vecdot` / `_mapfoldl`), vector updates
// are elementwise `u - c q`, and `Q' * Q` is the fused muladd chain of the StaticArrays product. With Real = double
// the results are bit-identical to the CPU oracle's restatement.
#pragma once

#include "cl_math.cuh"

namespace cl {

enum { QR_OK = 0, QR_PIVOT = 1, QR_PASSES = 2 };
constexpr int MAX_PASSES = 4;

struct QRRes { int count, status, column; };

template <int N, typename T>
__device__ __forceinline__ T dotv(const T* a, const T* b) {
    T s = a[0] * b[0];
#pragma unroll
    for (int i = 1; i < N; ++i) s = s + a[i] * b[i];
    return s;
}

// Gram-Schmidt family, orthonormalize.jl:38-105 (ALG = CL_QR_CGS, CL_QR_MGS or CL_QR_RGS).
template <int ALG, int D, int K, typename T>
__device__ __forceinline__ QRRes orth_gs(const T* W, T* Q, T* R) {
#pragma unroll
    for (int l = 0; l < D * K; ++l) Q[l] = T(0);
#pragma unroll
    for (int l = 0; l < K * K; ++l) R[l] = T(0);
    QRRes res{1, QR_OK, 0};
#pragma unroll
    for (int m = 0; m < K; ++m) {
        const T* w = W + m * D;
        T u[D];
        T r[K];
#pragma unroll
        for (int i = 0; i < K; ++i) r[i] = T(0);
#pragma unroll
        for (int i = 0; i < D; ++i) u[i] = w[i];
        int passes = 1;
        if (ALG == CL_QR_CGS || ALG == CL_QR_MGS) {
#pragma unroll
            for (int i = 0; i < m; ++i) {
                const T* qi = Q + i * D;
                const T c = dotv<D>(qi, ALG == CL_QR_CGS ? w : u);
                r[i] = c;
#pragma unroll
                for (int l = 0; l < D; ++l) u[l] = u[l] - c * qi[l];
            }
        } else {
            const T eta = T(1) / sqrt(T(2));
            T nold = nrm<D>(w);
            passes = 0;
            for (;;) {
                passes += 1;
                T vold[D];
#pragma unroll
                for (int l = 0; l < D; ++l) vold[l] = u[l];
#pragma unroll
                for (int i = 0; i < m; ++i) {
                    const T* qi = Q + i * D;
                    const T c = dotv<D>(qi, vold);
                    r[i] = r[i] + c;
#pragma unroll
                    for (int l = 0; l < D; ++l) u[l] = u[l] - c * qi[l];
                }
                const T nnew = nrm<D>(u);
                if (nnew >= nold * eta || !(isfin(nnew) && nnew > T(0))) break;
                if (passes == MAX_PASSES) { passes = MAX_PASSES + 1; break; }
                nold = nnew;
            }
        }
        const T gamma = nrm<D>(u);
#pragma unroll
        for (int i = 0; i < K; ++i) R[i + m * K] = i < m ? r[i] : (i == m ? gamma : T(0));
        if (passes > MAX_PASSES) { res.status = QR_PASSES; res.column = m + 1; }
        else if (!(isfin(gamma) && gamma > T(0))) { res.status = QR_PIVOT; res.column = m + 1; }
        if (res.status != QR_OK) break;
#pragma unroll
        for (int l = 0; l < D; ++l) Q[l + m * D] = dv(u[l], gamma);
        res.count = passes > res.count ? passes : res.count;
    }
    return res;
}

// _reflect (householder.jl:30-34) on a D x MC matrix.
template <int D, int MC, typename T>
__device__ __forceinline__ void hh_reflect(T* A, const T* u) {
    T w[MC];
#pragma unroll
    for (int l = 0; l < MC; ++l) w[l] = dotv<D>(u, A + l * D);
#pragma unroll
    for (int l = 0; l < MC; ++l)
#pragma unroll
        for (int i = 0; i < D; ++i) A[i + l * D] = A[i + l * D] - (T(2) * u[i]) * w[l];
}

// _hh_sweep with _reflector (householder.jl:19-50).
template <int D, int MC, int K, typename T>
__device__ __forceinline__ int hh_sweep(T* A, T* U) {
    constexpr int NREF = K < D ? K : K - 1;
    int count = 0;
#pragma unroll
    for (int l = 0; l < D * K; ++l) U[l] = T(0);
#pragma unroll
    for (int j = 0; j < NREF; ++j) {
        T a[D];
#pragma unroll
        for (int i = 0; i < D; ++i) a[i] = i >= j ? A[i + j * D] : T(0);
        const T c = nrm<D>(a);
        T rho;
        if (isfin(c) && c > T(0)) {
            const T s = a[j] < T(0) ? T(-1) : T(1);
            a[j] = a[j] + s * c;
            const T nv = nrm<D>(a);
            T u[D];
#pragma unroll
            for (int i = 0; i < D; ++i) u[i] = dv(a[i], nv);
            rho = -s * c;
            hh_reflect<D, MC>(A, u);
#pragma unroll
            for (int i = 0; i < D; ++i) U[i + j * D] = u[i];
            count += 1;
        } else {
            rho = c;
        }
        A[j + j * D] = rho;
    }
    return count;
}

// _finish (householder.jl:66-75). A has leading dimension LD.
template <int D, int K, int LD, typename T>
__device__ __forceinline__ QRRes hh_finish(T* Q, const T* A, int count, T* R) {
    T sg[K];
#pragma unroll
    for (int j = 0; j < K; ++j) sg[j] = A[j + j * LD] < T(0) ? T(-1) : T(1);
#pragma unroll
    for (int j = 0; j < K; ++j)
#pragma unroll
        for (int i = 0; i < K; ++i) R[i + j * K] = i > j ? T(0) : sg[i] * A[i + j * LD];
#pragma unroll
    for (int j = 0; j < K; ++j)
#pragma unroll
        for (int i = 0; i < D; ++i) Q[i + j * D] = Q[i + j * D] * sg[j];
    QRRes res{count, QR_OK, 0};
#pragma unroll
    for (int j = K - 1; j >= 0; --j) {   // the first failing pivot wins
        const T p = R[j + j * K];
        if (!(isfin(p) && p > T(0))) { res.status = QR_PIVOT; res.column = j + 1; }
    }
    return res;
}

template <int D, int K, typename T>
__device__ __forceinline__ QRRes orth_householder(const T* W, T* Q, T* R) {   // householder.jl:77-80
    T A[D * K], U[D * K];
#pragma unroll
    for (int l = 0; l < D * K; ++l) A[l] = W[l];
    const int count = hh_sweep<D, K, K>(A, U);
#pragma unroll
    for (int l = 0; l < D * K; ++l) Q[l] = (l % D) == (l / D) ? T(1) : T(0);
    constexpr int NREF = K < D ? K : K - 1;
#pragma unroll
    for (int j = NREF - 1; j >= 0; --j) hh_reflect<D, K>(Q, U + j * D);
    return hh_finish<D, K, D>(Q, A, count, R);
}

template <int D, int K, typename T>
__device__ __forceinline__ QRRes orth_augmented(const T* W, T* Q, T* R) {     // householder.jl:83-90
    constexpr int MC = K + D;
    T A[D * MC], U[D * K];
#pragma unroll
    for (int l = 0; l < D * MC; ++l) {
        const int i = l % D, j = l / D;
        A[l] = l < D * K ? W[l] : (i == j - K ? T(1) : T(0));
    }
    const int count = hh_sweep<D, MC, K>(A, U);
#pragma unroll
    for (int b = 0; b < K; ++b)
#pragma unroll
        for (int a = 0; a < D; ++a) Q[a + b * D] = A[b + (K + a) * D];
    return hh_finish<D, K, D>(Q, A, count, R);
}

template <int D, int K, typename T>
__device__ __forceinline__ QRRes orth_givens(const T* W, T* Q, T* R) {        // householder.jl:94-123
    constexpr int WD = K + D;
    T rows[D][WD];
#pragma unroll
    for (int i = 0; i < D; ++i)
#pragma unroll
        for (int l = 0; l < WD; ++l) rows[i][l] = l < K ? W[i + l * D] : (l - K == i ? T(1) : T(0));
    int count = 0;
    constexpr int J = K < D - 1 ? K : D - 1;
#pragma unroll
    for (int j = 0; j < J; ++j)
#pragma unroll
        for (int i = D - 1; i >= j + 1; --i) {
            const T ab[2] = {rows[i - 1][j], rows[i][j]};
            const T rho = nrm<2>(ab);
            if (isfin(rho) && rho > T(0)) {
                const T c = dv(ab[0], rho), s = dv(ab[1], rho);
#pragma unroll
                for (int l = 0; l < WD; ++l) {
                    const T ra = rows[i - 1][l], rb = rows[i][l];
                    rows[i - 1][l] = c * ra + s * rb;
                    rows[i][l] = c * rb - s * ra;
                }
                rows[i - 1][j] = rho;
                rows[i][j] = T(0);
                count += 1;
            }
        }
    T R0[K * K];
#pragma unroll
    for (int j = 0; j < K; ++j)
#pragma unroll
        for (int i = 0; i < K; ++i) R0[i + j * K] = i > j ? T(0) : rows[i][j];
#pragma unroll
    for (int b = 0; b < K; ++b)
#pragma unroll
        for (int a = 0; a < D; ++a) Q[a + b * D] = rows[b][K + a];
    return hh_finish<D, K, K>(Q, R0, count, R);
}

template <int ALG, int D, int K, typename T>
__device__ __forceinline__ QRRes orthonormalize(const T* W, T* Q, T* R) {
    if (ALG == CL_QR_HOUSEHOLDER) return orth_householder<D, K>(W, Q, R);
    if (ALG == CL_QR_AUGMENTED) return orth_augmented<D, K>(W, Q, R);
    if (ALG == CL_QR_GIVENS) return orth_givens<D, K>(W, Q, R);
    return orth_gs<ALG, D, K>(W, Q, R);
}

// window_Gw (orthonormalize.jl:112-127).
template <int K, typename T>
__device__ __forceinline__ T window_Gw(const T* R0) {
    T R[K * K];
    T m = fabs(R0[0]);
#pragma unroll
    for (int l = 1; l < K * K; ++l) m = mx(m, static_cast<T>(fabs(R0[l])));
    // T(1e100) is Inf and T(1e-100) is 0 in Float32, so the rescale never fires there (as in the reference).
    bool rescale = false;
    if constexpr (sizeof(T) == 8) rescale = (m > T(1e100) || m < T(1e-100)) && isfin(m) && m > T(0);
#pragma unroll
    for (int l = 0; l < K * K; ++l) R[l] = rescale ? dv(R0[l], m) : R0[l];
    T Ri[K * K];
#pragma unroll
    for (int l = 0; l < K * K; ++l) Ri[l] = T(0);
#pragma unroll
    for (int j = 0; j < K; ++j) {
        Ri[j + j * K] = dv(T(1), R[j + j * K]);
#pragma unroll
        for (int i = j - 1; i >= 0; --i) {
            T s = T(0);
#pragma unroll
            for (int l = i + 1; l <= j; ++l) s = s + R[i + l * K] * Ri[l + j * K];
            Ri[i + j * K] = dv(-s, R[i + i * K]);
        }
    }
    T a = R[0] * R[0], b = Ri[0] * Ri[0];
#pragma unroll
    for (int l = 1; l < K * K; ++l) { a = a + R[l] * R[l]; b = b + Ri[l] * Ri[l]; }
    return sqt(a) * sqt(b);
}

// _G_from_Gw (orthonormalize.jl:130-132).
template <int K, typename T>
__device__ __forceinline__ T G_from_Gw(T Gw) {
    if (K == 1) return T(1);
    if (K == 2) return (Gw + sqrt(jl_max(Gw * Gw - T(4), T(0)))) / T(2);
    return Gw;
}

// orth_loss (qr_spectrum.jl:4): maximum(abs, Q'Q - I) with Q'Q the fused StaticArrays product. Q'Q is symmetric bit
// for bit (each entry's fma chain has the same operands in the same order, and a*b == b*a), so the maximum over the
// upper triangle is the maximum over the matrix.
template <int D, int K, typename T>
__device__ __forceinline__ T orth_loss(const T* Q) {
    T m = T(0);
#pragma unroll
    for (int j = 0; j < K; ++j)
#pragma unroll
        for (int i = 0; i <= j; ++i) {
            T acc = Q[i * D] * Q[j * D];
#pragma unroll
            for (int q = 1; q < D; ++q) acc = fma(Q[q + i * D], Q[q + j * D], acc);
            if (i == j) acc = acc - T(1);
            const T a = fabs(acc);
            m = (i == 0 && j == 0) ? a : mx(m, a);
        }
    return m;
}

}  // namespace cl
