// oracle/oracle_capi.cpp -- TEST INFRASTRUCTURE (the CPU oracle). Only tests/, __graft_entry__.smoke() and the
// cpu_baseline / reference legs of bench.py load liboracle.so; the product never does.
//
// C entry points of the oracle. `oracle_propagate` is the serial per-orbit body of the reference
// (`_orbit_body`, src/Tangent/orbit.jl:44-60, driven as `_orbit_kernel!` drives it, src/Tangent/propagate.jl:32-50,
// including the carried-state relaunch n0 > 0), run over orbits on a pool of std::threads that take chunks of orbits from an atomic counter; orbits are independent, so the result
// does not depend on the thread count (propagate.jl:272-273). It takes the same cl_run / cl_buffers as
// libchaoslab_b200 (orbit-major host layout only).
#include <algorithm>
#include <atomic>
#include <thread>
#include <cstdio>
#include <cstring>
#include <limits>
#include <vector>

#include "oracle.hpp"

using namespace orc;

namespace {

constexpr int8_t STATUS_OK = 0, STATUS_STATE = 1, STATUS_W = 2, STATUS_REDUCER = 3;   // orbit.jl:1

int64_t frame_state_bytes(const cl_frame& f) {
    int64_t b = 0;
    for (int r = 0; r < f.n_reducers; ++r) b += state_bytes_of(f.reducers[r], f.k);
    return b;
}

// _status, orbit.jl:3: all(isfinite, x) ? (all(isfinite, W) ? OK : W) : STATE
int8_t status_of(const double* x, int s, const double* W, int dk) {
    for (int i = 0; i < s; ++i) if (!isfin(x[i])) return STATUS_STATE;
    for (int i = 0; i < dk; ++i) if (!isfin(W[i])) return STATUS_W;
    return STATUS_OK;
}

constexpr int8_t STATUS_ESCAPED = 4;

// max_j |p_j| over the momenta (second half of the state; (x, p) for the standard map)
double max_abs_p(const double* x, int d) {
    double m = std::fabs(x[d / 2]);
    for (int j = d / 2 + 1; j < d; ++j) m = std::fmax(m, std::fabs(x[j]));
    return m;
}

// One orbit. Ensembles pass a per-orbit K (Kp), length (Np) and the escape bound: the orbit then stops after the
// first handoff at which max |p_j| > escape with code 4, its records those of the run with N = that handoff.
template <int MM>
void run_orbit(const cl_run& run0, int64_t i, const cl_buffers& b, const double* Kp = nullptr,
               const int64_t* Np = nullptr, double escape = 0.0) {
    cl_run run = run0;
    if (Kp) run.sys.K = Kp[i];
    if (Np) { run.N = Np[i]; run.steps = 0; }
    const int d = run.d, s = run.s, nf = run.n_frames;
    const int64_t n0 = run.n0;
    const int64_t steps = run.steps > 0 ? run.steps : run.N - n0;
    double x[2 * CL_MAX_DIM];   // the wrapped maps carry a winding count per coordinate
    double W[CL_MAX_FRAMES][CL_MAX_DIM * CL_MAX_K];
    std::vector<uint8_t> st[CL_MAX_FRAMES];
    bool alive[CL_MAX_FRAMES];
    int8_t code[CL_MAX_FRAMES];
    int64_t hstep[CL_MAX_FRAMES];
    // A chain (GALI, SALI) with k > 2 holds the SALI record of a separate k = 2 run on the same orbit and the first
    // two columns of W0: that run's own frame is carried here and evolved by the same tangent products.
    double Ws[CL_MAX_FRAMES][CL_MAX_DIM * 2];
    int sali_slot[CL_MAX_FRAMES];
    const double* xin = (n0 == 0 && b.x0) ? b.x0 : b.x;
    std::memcpy(x, xin + i * s, sizeof(double) * s);
    bool any = false;
    for (int f = 0; f < nf; ++f) {
        const int k = run.frames[f].k;
        const int64_t sb = frame_state_bytes(run.frames[f]);
        st[f].assign(static_cast<size_t>(sb), 0);
        if (n0 == 0) {
            if (b.W0[f]) std::memcpy(W[f], b.W0[f] + i * d * k, sizeof(double) * d * k);
            else seeded_frame<MM>(run.seed, run.orbit_base + i + 1, d, k, W[f]);
            code[f] = STATUS_OK;
            alive[f] = true;
        } else {
            std::memcpy(W[f], b.W[f] + i * d * k, sizeof(double) * d * k);
            if (sb) std::memcpy(st[f].data(), static_cast<const uint8_t*>(b.states[f]) + i * sb, sb);
            code[f] = b.code[f][i];
            hstep[f] = b.hstep[f] ? b.hstep[f][i] : 0;
            alive[f] = code[f] == STATUS_OK;   // a failed orbit keeps its status and step (propagate.jl:34)
        }
        any = any || alive[f];
        sali_slot[f] = -1;
        const cl_frame& fr = run.frames[f];
        for (int r = 1; r < fr.n_reducers; ++r)
            if (fr.reducers[r].kind == CL_RED_SALI && fr.reducers[r - 1].kind == CL_RED_GALI && fr.k > 2) sali_slot[f] = r;
        // the separate run's frame: W0's first two columns (carried launches restore them from the GALI frame's
        // unit columns, which equal the SALI run's frame at every handoff)
        if (sali_slot[f] >= 0) std::memcpy(Ws[f], W[f], sizeof(double) * d * 2);
    }
    if (!any) return;   // frozen: nothing is written

    Systems<MM> sysf;
    (void)sysf;
    Chain<MM> chain{run.sys.n_sites, run.sys.K, run.sys.eps, run.sys.ring != 0};
    Gauss3 gauss(run.sys.gauss_maxiter, run.sys.gauss_tol);
    const SplitHH split = SplitHH::of(run.sys);
    int64_t n = n0;
    bool escaped = false;
    const int tau = run.tau;
    const int64_t handoffs = steps / tau;
    for (int64_t h = 0; h < handoffs; ++h) {
        for (int t = 0; t < tau; ++t) {
            if (run.sys.kind == CL_SYS_CHAIN || run.sys.kind == CL_SYS_WRAPPED_CHAIN) {
                double g[CL_MAX_DIM / 2], gl[CL_MAX_DIM / 2], gr[CL_MAX_DIM / 2];
                chain.band(x, g, gl, gr);
                for (int f = 0; f < nf; ++f) {
                    if (!alive[f]) continue;
                    chain.apply(g, gl, gr, W[f], run.frames[f].k);
                    if (sali_slot[f] >= 0) chain.apply(g, gl, gr, Ws[f], 2);
                }
                if (run.sys.kind == CL_SYS_WRAPPED_CHAIN) chain.forward_wrapped(x);
                else chain.forward(x);
            } else {
                double M[CL_MAX_DIM * CL_MAX_DIM];
                switch (run.sys.kind) {
                    case CL_SYS_STANDARD: Systems<MM>::standard(run.sys.K, x, M); break;
                    case CL_SYS_WRAPPED_STANDARD: Systems<MM>::wrapped(run.sys.K, x, M); break;
                    case CL_SYS_FROESCHLE: Systems<MM>::froeschle(run.sys.nu, run.sys.kappa, run.sys.mu, x, M); break;
                    case CL_SYS_WRAPPED_FROESCHLE:
                        Systems<MM>::wrapped_froeschle(run.sys.nu, run.sys.kappa, run.sys.mu, x, M);
                        break;
                    case CL_SYS_LINEAR: Systems<MM>::linear(run.sys.A, d, x, M); break;
                    case CL_SYS_HH_GAUSS: gauss.step(x, run.sys.dt, M); break;
                    case CL_SYS_HH_SPLIT: split.step(x, run.sys.dt, M); break;
                }
                for (int f = 0; f < nf; ++f) {
                    if (!alive[f]) continue;
                    double Wn[CL_MAX_DIM * CL_MAX_K];
                    fused_product(M, W[f], Wn, d, d, run.frames[f].k);
                    std::memcpy(W[f], Wn, sizeof(double) * d * run.frames[f].k);
                    if (sali_slot[f] >= 0) {
                        fused_product(M, Ws[f], Wn, d, d, 2);
                        std::memcpy(Ws[f], Wn, sizeof(double) * d * 2);
                    }
                }
            }
        }
        n += tau;
        bool still = false;
        for (int f = 0; f < nf; ++f) {
            if (!alive[f]) continue;
            const cl_frame& fr = run.frames[f];
            const int8_t c = status_of(x, s, W[f], d * fr.k);
            if (c != STATUS_OK) { code[f] = c; hstep[f] = n; alive[f] = false; continue; }
            // _apply (orbit.jl:23-28): every reducer runs, each on the W the one before returned
            uint8_t* p = st[f].data();
            for (int r = 0; r < fr.n_reducers; ++r) {
                if (r == sali_slot[f]) Reducers<MM>::step(fr.reducers[r], p, n, Ws[f], d, 2);
                else Reducers<MM>::step(fr.reducers[r], p, n, W[f], d, fr.k);
                p += state_bytes_of(fr.reducers[r], fr.k);
            }
            p = st[f].data();
            bool failed = false;
            for (int r = 0; r < fr.n_reducers; ++r) {
                failed = failed || Reducers<MM>::failed(fr.reducers[r], p, fr.k);
                p += state_bytes_of(fr.reducers[r], fr.k);
            }
            if (failed) { code[f] = STATUS_REDUCER; hstep[f] = n; alive[f] = false; continue; }
            still = true;
        }
        if (!still) break;
        if (escape > 0.0 && max_abs_p(x, d) > escape) { escaped = true; break; }
    }
    for (int f = 0; f < nf; ++f) {
        if (alive[f]) {   // orbit.jl:58: the final status check runs only at step N (here: N or the escape handoff)
            const int8_t c = status_of(x, s, W[f], d * run.frames[f].k);
            code[f] = escaped ? (c == STATUS_OK ? STATUS_ESCAPED : c) : (n == run.N ? c : STATUS_OK);
            hstep[f] = n;
        }
    }
    std::memcpy(b.x + i * s, x, sizeof(double) * s);
    for (int f = 0; f < nf; ++f) {
        const int k = run.frames[f].k;
        const int64_t sb = frame_state_bytes(run.frames[f]);
        const bool frozen_before = n0 > 0 && b.code[f][i] != STATUS_OK;
        if (frozen_before) continue;
        std::memcpy(b.W[f] + i * d * k, W[f], sizeof(double) * d * k);
        if (sb) std::memcpy(static_cast<uint8_t*>(b.states[f]) + i * sb, st[f].data(), sb);
        b.code[f][i] = code[f];
        if (b.hstep[f]) b.hstep[f][i] = hstep[f];
    }
}

// ---- the two-trajectory estimator (src/Lyapunov/two_trajectory.jl:31-80, separation.jl) ------------------------
// forward of the run's system (the tangent the system computes alongside is dropped)
template <int MM>
void forward_only(const cl_run& run, const Chain<MM>& chain, Gauss3& gauss, const SplitHH& split, double* x) {
    double M[CL_MAX_DIM * CL_MAX_DIM];
    switch (run.sys.kind) {
        case CL_SYS_STANDARD: Systems<MM>::standard(run.sys.K, x, M); break;
        case CL_SYS_WRAPPED_STANDARD: Systems<MM>::wrapped(run.sys.K, x, M); break;
        case CL_SYS_FROESCHLE: Systems<MM>::froeschle(run.sys.nu, run.sys.kappa, run.sys.mu, x, M); break;
        case CL_SYS_LINEAR: Systems<MM>::linear(run.sys.A, run.d, x, M); break;
        case CL_SYS_HH_GAUSS: gauss.step(x, run.sys.dt, M); break;
        case CL_SYS_HH_SPLIT: split.forward(x, run.sys.dt); break;
        case CL_SYS_CHAIN: {
            double g[CL_MAX_DIM / 2], gl[CL_MAX_DIM / 2], gr[CL_MAX_DIM / 2];
            chain.band(x, g, gl, gr);
            chain.forward(x);
            break;
        }
    }
}
// separation: y - x on lifted states; WrappedStandardMap: the minimal image in (-pi, pi] of both coordinates
void shadow_separation(const cl_run& run, const double* x, const double* y, double* delta) {
    if (run.sys.kind == CL_SYS_WRAPPED_STANDARD) {
        const double tp = 2 * jl_pi(), h = tp / 2;
        for (int i = 0; i < 2; ++i) {
            const double u = y[i] - x[i];
            delta[i] = u > h ? u - tp : (u <= -h ? u + tp : u);
        }
    } else {
        for (int i = 0; i < run.d; ++i) delta[i] = y[i] - x[i];
    }
}
// displaced: x + delta; WrappedStandardMap: both coordinates reduced, the reduction counts added to x's
void shadow_displaced(const cl_run& run, const double* x, const double* delta, double* y) {
    if (run.sys.kind == CL_SYS_WRAPPED_STANDARD) {
        const double tp = 2 * jl_pi();
        double xr, a, pr, b;
        wrap_reduce(x[0] + delta[0], tp, &xr, &a);
        wrap_reduce(x[1] + delta[1], tp, &pr, &b);
        y[0] = xr; y[1] = pr; y[2] = x[2] + a; y[3] = x[3] + b;
    } else {
        for (int i = 0; i < run.d; ++i) y[i] = x[i] + delta[i];
    }
}
void shadow_store(uint8_t* e, int s, const double* x, const double* y, CS acc, double dprev, int8_t code, int64_t step,
                  double value) {
    std::memset(e, 0, 8 * (2 * s + 6));
    std::memcpy(e, x, 8 * s);
    std::memcpy(e + 8 * s, y, 8 * s);
    std::memcpy(e + 8 * (2 * s), &acc.s, 8);
    std::memcpy(e + 8 * (2 * s + 1), &acc.c, 8);
    std::memcpy(e + 8 * (2 * s + 2), &dprev, 8);
    std::memcpy(e + 8 * (2 * s + 3), &code, 1);
    std::memcpy(e + 8 * (2 * s + 4), &step, 8);
    std::memcpy(e + 8 * (2 * s + 5), &value, 8);
}
// One orbit's ShadowEnd in the oracle's hands: start (_shadow_start), load / store, body over a segment.
template <int MM>
struct ShOrb {
    const cl_run& run;
    double x[CL_MAX_DIM] = {}, y[CL_MAX_DIM] = {};
    CS acc{0.0, 0.0};
    double dprev = 0.0, value = 0.0;
    int8_t code = 0;
    int64_t step = 0;
    explicit ShOrb(const cl_run& r) : run(r) {}
    void start(int64_t i, const double* x0, const double* u0, double d0) {
        const int s = run.s, d = run.d;
        double delta[CL_MAX_DIM] = {}, u[CL_MAX_DIM] = {};
        std::memcpy(x, x0 + i * s, 8 * s);
        if (u0) std::memcpy(u, u0 + i * d, 8 * d);
        else seeded_frame<MM>(run.seed, run.orbit_base + i + 1, d, 1, u);
        for (int c = 0; c < d; ++c) delta[c] = d0 * u[c];
        shadow_displaced(run, x, delta, y);
        shadow_separation(run, x, y, delta);
        dprev = safe_norm(delta, d);
        code = !(std::isfinite(dprev) && dprev > 0) ? 2 : (dprev < d0 / 2 || dprev > 2 * d0 ? 3 : 0);
        step = 0;
        value = dprev;
    }
    void load(const uint8_t* e) {
        const int s = run.s;
        std::memcpy(x, e, 8 * s);
        std::memcpy(y, e + 8 * s, 8 * s);
        std::memcpy(&acc.s, e + 8 * (2 * s), 8);
        std::memcpy(&acc.c, e + 8 * (2 * s + 1), 8);
        std::memcpy(&dprev, e + 8 * (2 * s + 2), 8);
        std::memcpy(&code, e + 8 * (2 * s + 3), 1);
        std::memcpy(&step, e + 8 * (2 * s + 4), 8);
        std::memcpy(&value, e + 8 * (2 * s + 5), 8);
    }
    void store(uint8_t* e) const { shadow_store(e, run.s, x, y, acc, dprev, code, step, value); }
    void body(int64_t n, int64_t steps, double d0) {
        using Mth = Math<MM>;
        const int s = run.s, d = run.d;
        const Chain<MM> chain{run.sys.n_sites, run.sys.K, run.sys.eps, run.sys.ring != 0};
        Gauss3 gauss(run.sys.gauss_maxiter, run.sys.gauss_tol);
        const SplitHH split = SplitHH::of(run.sys);
        double delta[CL_MAX_DIM] = {};
        for (int64_t h = 0; h < steps / run.tau; ++h) {
            for (int t = 0; t < run.tau; ++t) {
                forward_only<MM>(run, chain, gauss, split, x);
                forward_only<MM>(run, chain, gauss, split, y);
            }
            n += run.tau;
            // _first_bad_value: the first non-finite entry of x, else of y
            bool fin = true;
            double bad = 0.0;
            for (int c = 0; c < s && fin; ++c) if (!std::isfinite(x[c])) { fin = false; bad = x[c]; }
            for (int c = 0; c < s && fin; ++c) if (!std::isfinite(y[c])) { fin = false; bad = y[c]; }
            if (!fin) { code = 1; step = n; value = bad; return; }
            shadow_separation(run, x, y, delta);
            const double dd = safe_norm(delta, d);
            if (!(std::isfinite(dd) && dd > 0)) { code = 2; step = n; value = dd; return; }
            acc = cs_add(acc, Mth::log(dd / dprev));
            const double f = d0 / dd;
            for (int c = 0; c < d; ++c) delta[c] = delta[c] * f;
            shadow_displaced(run, x, delta, y);
            shadow_separation(run, x, y, delta);
            dprev = safe_norm(delta, d);
            if (!(dprev >= d0 / 2 && dprev <= 2 * d0)) {
                code = (std::isfinite(dprev) && dprev > 0) ? 3 : 2;
                step = n;
                value = dprev;
                return;
            }
        }
        code = 0;
        step = n;
        value = dprev;
    }
};

template <int MM>
void shadow_orbit(const cl_run& run, int64_t i, const double* x0, const double* u0, uint8_t* ends, double d0,
                  int64_t n0, int64_t steps, const int64_t* grid = nullptr, int n_grid = 0, double* R = nullptr,
                  int64_t* fail = nullptr) {
    const int s = run.s;
    uint8_t* e = ends + i * 8 * (2 * s + 6);
    ShOrb<MM> o(run);
    if (n0 == 0) {
        o.start(i, x0, u0, d0);
        if (!grid && o.code != 0) { o.store(e); return; }
    } else {
        o.load(e);
        if (o.code != 0) return;
    }
    if (!grid) {
        o.body(n0, steps, d0);
        o.store(e);
        return;
    }
    // _shadow_record_kernel! (src/Experiments/run_device.jl:80-100)
    const int ncol = 1 + 7 + s;
    int glo = 0;
    while (glo < n_grid && grid[glo] <= n0) ++glo;
    int ghi = glo - 1;
    while (ghi + 1 < n_grid && grid[ghi + 1] <= n0 + steps) ++ghi;
    int64_t n = n0;
    double* Ri = R + i * static_cast<int64_t>(ncol) * n_grid;
    for (int g = glo; g <= ghi; ++g) {
        if (o.code == 0) o.body(n, grid[g] - n, d0);
        if (o.code != 0) { fail[i] = g + 1; o.store(e); return; }
        n = grid[g];
        double* row = Ri + static_cast<int64_t>(g) * ncol;
        row[0] = (o.acc.s + o.acc.c) / static_cast<double>(grid[g]);
        for (int j = 0; j < s; ++j) row[8 + j] = o.x[j];
    }
    if (o.code == 0 && n < n0 + steps) {
        o.body(n, n0 + steps - n, d0);
        if (o.code != 0) fail[i] = ghi + 2;
    } else if (o.code != 0 && glo > ghi) {
        fail[i] = ghi + 2;
    }
    o.store(e);
}

// ---- the study recorder (src/Experiments/run_device.jl:43-78, run_record.jl:24-40) ----------------------------
// map step of a recorder system: the tangent M at x (column-major 2 x 2), then x advanced
template <int MM>
void rec_map(const cl_run& run, double* x, double* M) {
    switch (run.sys.kind) {
        case CL_SYS_STANDARD: Systems<MM>::standard(run.sys.K, x, M); break;
        case CL_SYS_WRAPPED_STANDARD: Systems<MM>::wrapped(run.sys.K, x, M); break;
        case CL_SYS_LINEAR: Systems<MM>::linear(run.sys.A, run.d, x, M); break;
    }
}
// RunMonitor's step: |det M - 1|, max|M' Omega M - Omega| (StaticArrays products, the fused chain), max|M|
template <int MM>
void rec_monitor(const cl_run& run, const double* x, double* mon) {
    double xc[CL_MAX_DIM], M[4];
    std::memcpy(xc, x, sizeof(double) * run.s);
    rec_map<MM>(run, xc, M);
    const double edet = std::fabs((M[0] * M[3] - M[2] * M[1]) - 1.0);
    const double Om[4] = {0.0, -1.0, 1.0, 0.0};
    double P[4], Q[4];
    for (int j = 0; j < 2; ++j)
        for (int i = 0; i < 2; ++i) P[i + 2 * j] = std::fma(M[1 + 2 * i], Om[1 + 2 * j], M[2 * i] * Om[2 * j]);
    for (int j = 0; j < 2; ++j)
        for (int i = 0; i < 2; ++i) Q[i + 2 * j] = std::fma(P[i + 2], M[1 + 2 * j], P[i] * M[2 * j]);
    double es = std::fabs(Q[0] - Om[0]);
    for (int l = 1; l < 4; ++l) es = jl_max(es, std::fabs(Q[l] - Om[l]));
    double mm = std::fabs(M[0]);
    for (int l = 1; l < 4; ++l) mm = jl_max(mm, std::fabs(M[l]));
    mon[0] = jl_max(mon[0], edet);
    mon[1] = jl_max(mon[1], es);
    mon[2] = jl_max(mon[2], mm);
}
// _orbit_body (orbit.jl:44-60) with the chain (estimator, monitor); est the estimator's bytes, mon its 3 doubles
template <int MM>
int8_t rec_body(const cl_run& run, double* x, double* W, uint8_t* est, double* mon, int64_t& n, int64_t steps) {
    const int d = run.d, k = run.frames[0].k, s = run.s;
    const cl_reducer& rd = run.frames[0].reducers[0];
    for (int64_t h = 0; h < steps / run.tau; ++h) {
        for (int t = 0; t < run.tau; ++t) {
            double M[4], Wn[4];
            rec_map<MM>(run, x, M);
            fused_product(M, W, Wn, d, d, k);
            std::memcpy(W, Wn, sizeof(double) * d * k);
        }
        n += run.tau;
        const int8_t c = status_of(x, s, W, d * k);
        if (c != STATUS_OK) return c;
        Reducers<MM>::step(rd, est, n, W, d, k);
        rec_monitor<MM>(run, x, mon);
        if (Reducers<MM>::failed(rd, est, k)) return STATUS_REDUCER;
    }
    return n == run.N ? status_of(x, s, W, d * k) : STATUS_OK;
}
template <int MM>
void rec_orbit(const cl_run& run, int64_t i, double* xs, double* Ws, uint8_t* sts, int8_t* code, int64_t* hstep,
               const int64_t* grid, int n_grid, double* R, int64_t* fail, int64_t n0, int64_t steps) {
    if (!(n0 == 0 || code[i] == STATUS_OK)) return;
    const int d = run.d, k = run.frames[0].k, s = run.s, ncol = k + 7 + s;
    const cl_reducer& rd = run.frames[0].reducers[0];
    const int64_t eb = state_bytes_of(rd, k), sb = eb + 24;
    double* x = xs + i * s;
    double* W = Ws + i * d * k;
    uint8_t* est = sts + i * sb;
    double mon[3];
    if (n0 == 0) { std::memset(est, 0, sb); mon[0] = mon[1] = mon[2] = 0.0; }
    else std::memcpy(mon, est + eb, 24);
    int64_t n = n0, h = n0;
    int8_t c = STATUS_OK;
    int glo = 0;
    while (glo < n_grid && grid[glo] <= n0) ++glo;
    int ghi = glo - 1;
    while (ghi + 1 < n_grid && grid[ghi + 1] <= n0 + steps) ++ghi;
    double* Ri = R + i * static_cast<int64_t>(ncol) * n_grid;
    for (int g = glo; g <= ghi; ++g) {
        c = rec_body<MM>(run, x, W, est, mon, n, grid[g] - n);
        h = n;
        if (c != STATUS_OK) { fail[i] = g + 1; break; }
        double lam[2] = {0.0, 0.0}, orth, gmax;
        int64_t sn;
        if (rd.kind == CL_RED_BENETTIN) {
            CS sum; std::memcpy(&sum, est, 16); std::memcpy(&sn, est + 16, 8);
            lam[0] = sn == 0 ? 0.0 : (sum.s + sum.c) / static_cast<double>(sn);
            orth = 0.0; gmax = 1.0;
        } else {
            CS sums[2]; std::memcpy(sums, est, 32); std::memcpy(&sn, est + 32, 8);
            std::memcpy(&gmax, est + 40, 8); std::memcpy(&orth, est + 48, 8);
            for (int j = 0; j < 2; ++j) lam[j] = sn == 0 ? 0.0 : (sums[j].s + sums[j].c) / static_cast<double>(sn);
        }
        double* row = Ri + static_cast<int64_t>(g) * ncol;
        for (int j = 0; j < k; ++j) row[j] = lam[j];
        row[k] = mon[0];
        row[k + 1] = mon[1];
        row[k + 2] = orth;
        if (k == 2) {
            const double sp = std::fabs(lam[0] + lam[1]);
            row[k + 3] = g > 0 ? jl_max(row[k + 3 - ncol], sp) : sp;
            row[k + 4] = g > 0 ? jl_max(row[k + 4 - ncol], sp) : sp;
        }
        row[k + 5] = gmax;
        row[k + 6] = mon[2];
        for (int j = 0; j < s; ++j) row[k + 7 + j] = x[j];
    }
    if (c == STATUS_OK && n < n0 + steps) {
        c = rec_body<MM>(run, x, W, est, mon, n, n0 + steps - n);
        h = n;
        if (c != STATUS_OK) fail[i] = ghi + 2;
    }
    std::memcpy(est + eb, mon, 24);
    code[i] = c;
    if (hstep) hstep[i] = h;
}

// ---- the indicator recorder, tangent and pair kinds (src/Experiments/run_indicator_device.jl:13-60) -------------
// _orbit_body (orbit.jl:44-60) with the chain (members..., RunMonitor): every member steps on the W the one before
// returned, then the monitor; a failure of any member stops the segment. `pair`: the stream is PairMap(sys)
// (src/Systems/pair.jl:9-68): the state (A; B) of two base states each advanced alone, the tangent acting block by
// block on the frame's rows (each block by the base's own product), the monitor reading orbit A
// (run_indicator_record.jl:6-10).
template <int MM>
int8_t ind_body(const cl_run& run, bool pair, double* x, double* W, uint8_t* st, double* mon, int64_t& n,
                int64_t steps) {
    const cl_frame& fr = run.frames[0];
    const int db = run.d, sb = run.s, k = fr.k;
    const int d = pair ? 2 * db : db, s = pair ? 2 * sb : sb;
    for (int64_t h = 0; h < steps / run.tau; ++h) {
        for (int t = 0; t < run.tau; ++t) {
            for (int half = 0; half < (pair ? 2 : 1); ++half) {
                double M[4], Wb[4], Wn[4];
                rec_map<MM>(run, x + half * sb, M);
                for (int j = 0; j < k; ++j)
                    for (int l = 0; l < db; ++l) Wb[l + db * j] = W[half * db + l + d * j];
                fused_product(M, Wb, Wn, db, db, k);
                for (int j = 0; j < k; ++j)
                    for (int l = 0; l < db; ++l) W[half * db + l + d * j] = Wn[l + db * j];
            }
        }
        n += run.tau;
        const int8_t c = status_of(x, s, W, d * k);
        if (c != STATUS_OK) return c;
        uint8_t* p = st;
        for (int r = 0; r < fr.n_reducers; ++r) {
            Reducers<MM>::step(fr.reducers[r], p, n, W, d, k);
            p += state_bytes_of(fr.reducers[r], k);
        }
        rec_monitor<MM>(run, x, mon);
        p = st;
        bool failed = false;
        for (int r = 0; r < fr.n_reducers; ++r) {
            failed = failed || Reducers<MM>::failed(fr.reducers[r], p, k);
            p += state_bytes_of(fr.reducers[r], k);
        }
        if (failed) return STATUS_REDUCER;
    }
    return n == run.N ? status_of(x, s, W, d * k) : STATUS_OK;
}
// megno_series (megno.jl:97-102): Y = 2 R1 / n, Ybar = Q / K, Ybar20 = (n / K) Q2 / n^3; zeros before the first handoff
void ind_megno_series(const MegnoSumsJ& m, int64_t n, int64_t K, double* out) {
    if (K == 0) { out[0] = out[1] = out[2] = 0.0; return; }
    const double tn = static_cast<double>(n);
    out[0] = 2 * (m.R1.s + m.R1.c) / tn;
    out[1] = (m.Q.s + m.Q.c) / static_cast<double>(K);
    out[2] = static_cast<double>(n / K) * (m.Q2.s + m.Q2.c) / (tn * tn * tn);
}
// _put! (run_indicator_record.jl:40-56) of one member from its state: SALI sali, L (sali.jl:62-66); FLI fli = fB,
// fli1 = f1 (fli.jl:91-94); MEGNO Y, Ybar, Ybar20 of column 1 then of column 2; RLI DL, RLI. Returns the columns
// written.
int ind_put(const cl_reducer& rd, const uint8_t* b, double* row) {
    switch (rd.kind) {
        case CL_RED_SALI: {
            SALIStateJ st; std::memcpy(&st, b, sizeof st);
            row[0] = st.sali;
            row[1] = st.n == 0 ? 0.0 : -((st.s1.s + st.s2.s) + (st.s1.c + st.s2.c));
            return 2;
        }
        case CL_RED_FLI: {
            FLIStateJ st; std::memcpy(&st, b, sizeof st);
            row[0] = st.fB;
            row[1] = st.f1;
            return 2;
        }
        case CL_RED_MEGNO: {
            MEGNOStateJ st; std::memcpy(&st, b, sizeof st);
            ind_megno_series(st.c1, st.n, st.K, row);
            ind_megno_series(st.c2, st.n, st.K, row + 3);
            return 6;
        }
        case CL_RED_RLI: {   // reducer_final (rli.jl:98-101): DL at the last handoff, RLI = Q / K; zeros before one
            RLIStateJ st; std::memcpy(&st, b, sizeof st);
            row[0] = st.K == 0 ? 0.0 : std::fabs((st.sB.s - st.sA.s) + (st.sB.c - st.sA.c)) / static_cast<double>(st.n);
            row[1] = st.K == 0 ? 0.0 : (st.Q.s + st.Q.c) / static_cast<double>(st.K);
            return 2;
        }
    }
    return 0;
}
int ind_cols(const cl_frame& fr) {
    int c = 0;
    for (int r = 0; r < fr.n_reducers; ++r) c += fr.reducers[r].kind == CL_RED_MEGNO ? 6 : 2;
    return c;
}
// _ind_series_kernel! (run_indicator_device.jl:31-60) for one orbit over one launch window
template <int MM>
void ind_orbit(const cl_run& run, bool pair, int64_t i, int ns, double* xs, double* Ws, uint8_t* sts, int8_t* code,
               int64_t* hstep, const int64_t* grid, int n_grid, double* R, int64_t* fail, int64_t n0, int64_t steps) {
    if (!(n0 == 0 || code[i] == STATUS_OK)) return;
    const cl_frame& fr = run.frames[0];
    const int d = pair ? 2 * run.d : run.d, k = fr.k, s = pair ? 2 * run.s : run.s, ncol = ind_cols(fr) + 3 + ns;
    const int64_t cb = frame_state_bytes(fr), sb = cb + 24;
    double* x = xs + i * s;
    double* W = Ws + i * d * k;
    uint8_t* st = sts + i * sb;
    double mon[3];
    if (n0 == 0) { std::memset(st, 0, sb); mon[0] = mon[1] = mon[2] = 0.0; }
    else std::memcpy(mon, st + cb, 24);
    int64_t n = n0, h = n0;
    int8_t c = STATUS_OK;
    int glo = 0;
    while (glo < n_grid && grid[glo] <= n0) ++glo;
    int ghi = glo - 1;
    while (ghi + 1 < n_grid && grid[ghi + 1] <= n0 + steps) ++ghi;
    double* Ri = R + i * static_cast<int64_t>(ncol) * n_grid;
    for (int g = glo; g <= ghi; ++g) {
        c = ind_body<MM>(run, pair, x, W, st, mon, n, grid[g] - n);
        h = n;
        if (c != STATUS_OK) { fail[i] = g + 1; break; }
        double* row = Ri + static_cast<int64_t>(g) * ncol;
        const uint8_t* p = st;
        int off = 0;
        for (int r = 0; r < fr.n_reducers; ++r) {
            off += ind_put(fr.reducers[r], p, row + off);
            p += state_bytes_of(fr.reducers[r], k);
        }
        row[off] = mon[0];
        row[off + 1] = mon[1];
        row[off + 2] = mon[2];
        for (int j = 0; j < ns; ++j) row[off + 3 + j] = x[j];
    }
    if (c == STATUS_OK && n < n0 + steps) {
        c = ind_body<MM>(run, pair, x, W, st, mon, n, n0 + steps - n);
        h = n;
        if (c != STATUS_OK) fail[i] = ghi + 2;
    }
    std::memcpy(st + cb, mon, 24);
    code[i] = c;
    if (hstep) hstep[i] = h;
}

// ---- the indicator recorder, window kinds (src/Experiments/run_indicator_device.jl:62-91) ------------------------
// Julia's x^n for n = 1..4 (Base.Math power by squaring with the error terms): x, x x, (x x) x, and for n = 4 the
// square of the square with both product errors folded in.
double jl_powi(double x, int n) {
    if (n == 1) return x;
    if (n == 2) return x * x;
    if (n == 3) return x * x * x;
    const double x2 = x * x, e2 = std::fma(x, x, -x2);
    const double err = (x2 * 2) * e2;
    const double x4 = x2 * x2, e4 = std::fma(x2, x2, -x4);
    return x4 + (e4 + err);
}
// _wb (naff_reducer.jl:13-17): birkhoff_weight(min(j, N - j) / N, p) = exp(-1 / (t^p (1 - t)^p)), 0 at the ends
template <int MM>
double wb_weight(int64_t j, int64_t N, int p) {
    const double t = static_cast<double>(std::min(j, N - j)) / static_cast<double>(N);
    if (t <= 0.0 || t >= 1.0) return 0.0;
    return Math<MM>::exp(-1.0 / (jl_powi(t, p) * jl_powi(1.0 - t, p)));
}
template <typename T> T fld(const uint8_t* b, int off) { T v; std::memcpy(&v, b + off, sizeof v); return v; }
template <typename T> void fst(uint8_t* b, int off, T v) { std::memcpy(b + off, &v, sizeof v); }
// _unit_scale (naff_reducer.jl:36-41)
void unit_scale(double& re, double& im) {
    const double m = jl_max(std::fabs(re), std::fabs(im));
    int e = 0;
    if (std::isfinite(m) && m > 0) {
        e = static_cast<int>((bits_of(m) >> 52) & 0x7ff) - 1023;
        e = std::min(1000, std::max(-1000, e));
    }
    const double sc = p_pow2(-e);
    re = re * sc;
    im = im * sc;
}
// _phase_inc (naff_reducer.jl:45-53): arg(z conj(zp)) by atan2, NaN if either sample is exactly 0
template <int MM>
double phase_inc(double pr, double pim, double zr, double zi) {
    if ((pr == 0.0 && pim == 0.0) || (zr == 0.0 && zi == 0.0)) return std::numeric_limits<double>::quiet_NaN();
    double wr = pr, wi = -pim;
    double rr = zr * wr - zi * wi, ri = zr * wi + zi * wr;
    const double sm = jl_max(std::fabs(rr), std::fabs(ri));
    if (!(sm > 1e-280 && sm < 1e280)) {
        unit_scale(zr, zi);
        unit_scale(pr, pim);
        wr = pr; wi = -pim;
        rr = zr * wr - zi * wi;
        ri = zr * wi + zi * wr;
    }
    return Math<MM>::atan2(ri, rr);
}
int64_t window_reader_bytes(const cl_window& w) {
    return w.kind == CL_WIN_PHASE_ADVANCE ? 64 * static_cast<int64_t>(w.n_windows) + 32
                                          : 16 + static_cast<int64_t>(w.n_windows) * (16 + 40 * w.n_observables);
}
// reducer_step of WeightedPhaseAdvance (naff_reducer.jl:194-207) on WPAState{Float64, H}
template <int MM>
void wpa_step(const cl_window& w, uint8_t* st, int64_t n, const double* x) {
    const int H = w.n_windows, tail = 64 * H;
    if (fld<int8_t>(st, tail + 30) != 0) return;
    const int kind = w.obs_kind[0], ia = w.obs_a[0] - 1, ib = w.obs_b[0];
    const double s1 = x[ia], s2 = kind == CL_OBS_PLANAR ? x[ib - 1] : (ib == 0 ? 0.0 : x[ib - 1]);
    if (!(std::isfinite(s1) && std::isfinite(s2))) {
        fst<int64_t>(st, tail + 16, n);
        fst<int8_t>(st, tail + 30, 1);
        return;
    }
    const int32_t s = fld<int32_t>(st, tail + 24);
    const int32_t h1 = s < 2147483647 ? s + 1 : s;
    if (s == 0) {
        fst(st, tail, s1); fst(st, tail + 8, s2); fst<int64_t>(st, tail + 16, n); fst<int32_t>(st, tail + 24, h1);
        return;
    }
    const double p1 = fld<double>(st, tail), p2 = fld<double>(st, tail + 8);
    const double pi_ = 3.141592653589793;   // _pi(one(Float64))
    const double d = kind == CL_OBS_PLANAR ? phase_inc<MM>(p1, p2, s1, s2) : (s1 - p1) + (2 * pi_) * (s2 - p2);
    const int64_t j = s - 1;
    int64_t maxwin = 0;
    for (int h = 0; h < H; ++h) maxwin = std::max<int64_t>(maxwin, w.window[h]);
    for (int h = 0; h < H; ++h) {   // _advance (:176-186), _accumulate (:66)
        const int64_t N = w.window[h];
        if (j >= 2 * N) continue;
        const int off = 64 * h + (j < N ? 0 : 32);
        const double wt = wb_weight<MM>(j < N ? j : j - N, N, w.birkhoff_order);
        if (wt == 0.0) continue;
        const CS A = cs_add(CS{fld<double>(st, off), fld<double>(st, off + 8)}, wt * d);
        const CS B = cs_add(CS{fld<double>(st, off + 16), fld<double>(st, off + 24)}, wt);
        fst(st, off, A.s); fst(st, off + 8, A.c); fst(st, off + 16, B.s); fst(st, off + 24, B.c);
    }
    const int16_t nw = fld<int16_t>(st, tail + 28);
    const bool flagged = kind == CL_OBS_PLANAR && std::fabs(d) > (9.0 * pi_) / 10.0 && s <= 2 * maxwin && nw < 32767;
    fst(st, tail, s1); fst(st, tail + 8, s2); fst<int64_t>(st, tail + 16, n); fst<int32_t>(st, tail + 24, h1);
    if (flagged) fst<int16_t>(st, tail + 28, static_cast<int16_t>(nw + 1));
}
// the observables of a Birkhoff reader (wbirkhoff.jl:51-56; IndCoordinate, run_indicator_chain.jl:23)
template <int MM>
double wb_observable(const cl_window& w, int k, const double* x) {
    const int ia = w.obs_a[k] - 1, ib = w.obs_b[k];
    switch (w.obs_kind[k]) {
        case CL_OBS_COS: return Math<MM>::cos(static_cast<double>(ib) * x[ia]);
        case CL_OBS_SIN: return Math<MM>::sin(static_cast<double>(ib) * x[ia]);
        case CL_OBS_LIFTED: return x[ia] + (2 * 3.141592653589793) * x[ib - 1];
        default: return x[ia];
    }
}
// reducer_step of WeightedBirkhoff (wbirkhoff_reducer.jl:72-84) on WBState{Float64, H, K}
template <int MM>
void wb_step(const cl_window& w, uint8_t* st, int64_t n, const double* x) {
    const int H = w.n_windows, K = w.n_observables, hb = 16 + 40 * K, tail = H * hb;
    if (fld<int16_t>(st, tail + 12) != 0) return;
    int64_t maxwin = 0;
    for (int h = 0; h < H; ++h) maxwin = std::max<int64_t>(maxwin, w.window[h]);
    const int32_t hand = fld<int32_t>(st, tail + 8);
    if (static_cast<int64_t>(hand) >= 2 * maxwin) {
        fst<int64_t>(st, tail, n);
        if (hand < 2147483647) fst<int32_t>(st, tail + 8, hand + 1);
        return;
    }
    double v[CL_MAX_OBSERVABLES];
    int bad = 0;
    for (int k = 0; k < K; ++k) {
        v[k] = wb_observable<MM>(w, k, x);
        if (bad == 0 && !std::isfinite(v[k])) bad = k + 1;
    }
    if (bad) {
        fst<int64_t>(st, tail, n);
        fst<int16_t>(st, tail + 12, static_cast<int16_t>(bad));
        return;
    }
    const int64_t j = hand;
    for (int h = 0; h < H; ++h) {   // _wb_advance (:56-62), _wb_sample (wbirkhoff.jl:86-90)
        const int64_t N = w.window[h];
        if (j >= 2 * N) continue;
        const int i = j >= N ? 1 : 0;
        const double wt = wb_weight<MM>(j - i * N, N, w.birkhoff_order);
        const int off = h * hb;
        if (i == 0 && wt != 0.0) {
            const CS B = cs_add(CS{fld<double>(st, off), fld<double>(st, off + 8)}, wt);
            fst(st, off, B.s); fst(st, off + 8, B.c);
        }
        for (int k = 0; k < K; ++k) {
            const int c = off + 16 + 40 * k;
            fst(st, c + 32, jl_max(fld<double>(st, c + 32), std::fabs(v[k])));
            if (wt == 0.0) continue;
            const int ai = c + 16 * i;
            const CS A = cs_add(CS{fld<double>(st, ai), fld<double>(st, ai + 8)}, wt * v[k]);
            fst(st, ai, A.s); fst(st, ai + 8, A.c);
        }
    }
    fst<int64_t>(st, tail, n);
    fst<int32_t>(st, tail + 8, j < 2147483647 ? static_cast<int32_t>(j + 1) : hand);
}
// _ind_window_kernel! (run_indicator_device.jl:62-91) for one orbit over one launch window
template <int MM>
void win_orbit(const cl_run& run, const cl_window& w, int64_t i, int ns, double* xs, uint8_t* sts, int8_t* code,
               int64_t* hstep, const int64_t* grid, int n_grid, double* R, int64_t* fail, int64_t n0, int64_t steps) {
    if (!(n0 == 0 || code[i] == STATUS_OK)) return;
    const int s = run.s, ncol = 3 + ns;
    const int64_t rb = window_reader_bytes(w), sb = 24 + rb;
    double* x = xs + i * s;
    uint8_t* st = sts + i * sb;
    double mon[3];
    if (n0 == 0) { std::memset(st, 0, sb); mon[0] = mon[1] = mon[2] = 0.0; }
    else std::memcpy(mon, st, 24);
    uint8_t* rs = st + 24;
    int g = 0;
    while (g < n_grid && grid[g] <= n0) ++g;
    int ghi = g - 1;
    while (ghi + 1 < n_grid && grid[ghi + 1] <= n0 + steps) ++ghi;
    double* Ri = R + i * static_cast<int64_t>(ncol) * n_grid;
    int64_t n = n0, h = n0;
    int8_t c = STATUS_OK;
    for (int64_t hh = 0; hh < steps / run.tau; ++hh) {
        double W[2] = {1.0, 0.0}, Wn[2], M[4];
        for (int t = 0; t < run.tau; ++t) {
            rec_map<MM>(run, x, M);
            fused_product(M, W, Wn, 2, 2, 1);
            W[0] = Wn[0]; W[1] = Wn[1];
        }
        const int64_t nn = n + run.tau;
        c = status_of(x, s, W, 2);
        if (c == STATUS_OK) {
            rec_monitor<MM>(run, x, mon);
            if (w.kind == CL_WIN_PHASE_ADVANCE) wpa_step<MM>(w, rs, nn, x);
            else wb_step<MM>(w, rs, nn, x);
            const bool failed = w.kind == CL_WIN_PHASE_ADVANCE ? fld<int8_t>(rs, 64 * w.n_windows + 30) != 0
                                                               : fld<int16_t>(rs, static_cast<int>(rb) - 4) != 0;
            if (failed) c = STATUS_REDUCER;
        }
        h = nn;
        if (c != STATUS_OK) { fail[i] = (g <= ghi ? g : ghi + 1) + 1; break; }
        n = nn;
        if (g <= ghi && n == grid[g]) {
            double* row = Ri + static_cast<int64_t>(g) * ncol;
            row[0] = mon[0]; row[1] = mon[1]; row[2] = mon[2];
            for (int j = 0; j < ns; ++j) row[3 + j] = x[j];
            ++g;
        }
    }
    std::memcpy(st, mon, 24);
    code[i] = c;
    if (hstep) hstep[i] = h;
}

}  // namespace

extern "C" {

int64_t oracle_state_bytes(const cl_run* run, int32_t f) { return frame_state_bytes(run->frames[f]); }

// Propagate n orbits on the CPU; math_mode 0 = portable functions, 1 = glibc; threads <= 0 = all.
int oracle_propagate(const cl_run* run, int64_t n, const cl_buffers* b, int32_t math_mode, int32_t threads) {
    if (run->N <= 0 || run->tau <= 0 || run->N % run->tau != 0) return CL_EINVAL;
    const int64_t steps = run->steps > 0 ? run->steps : run->N - run->n0;
    if (steps % run->tau != 0 || run->n0 + steps > run->N) return CL_EINVAL;
    if (run->n_frames < 1 || run->n_frames > CL_MAX_FRAMES) return CL_EINVAL;
    const int hw = static_cast<int>(std::max(1u, std::thread::hardware_concurrency()));
    const int nt = static_cast<int>(std::min<int64_t>(threads > 0 ? threads : hw, std::max<int64_t>(n, 1)));
    std::atomic<int64_t> next{0};
    auto worker = [&]() {
        for (;;) {
            const int64_t lo = next.fetch_add(16);
            if (lo >= n) return;
            const int64_t hi = std::min<int64_t>(lo + 16, n);
            for (int64_t i = lo; i < hi; ++i) {
                if (math_mode == MATH_LIBM) run_orbit<MATH_LIBM>(*run, i, *b);
                else run_orbit<MATH_PORTABLE>(*run, i, *b);
            }
        }
    };
    std::vector<std::thread> pool;
    for (int t = 1; t < nt; ++t) pool.emplace_back(worker);
    worker();
    for (auto& th : pool) th.join();
    return 0;
}

// A batched uneven ensemble class (one frame): per-orbit K (may be NULL), lengths (may be NULL), escape bound.
int oracle_ensemble(const cl_run* run, int64_t n, const cl_buffers* b, const double* K, const int64_t* N,
                    double escape, int32_t math_mode, int32_t threads) {
    if (run->n_frames != 1 || run->n0 != 0) return CL_EINVAL;
    const int hw = static_cast<int>(std::max(1u, std::thread::hardware_concurrency()));
    const int nt = static_cast<int>(std::min<int64_t>(threads > 0 ? threads : hw, std::max<int64_t>(n, 1)));
    std::atomic<int64_t> next{0};
    auto worker = [&]() {
        for (;;) {
            const int64_t lo = next.fetch_add(4);
            if (lo >= n) return;
            for (int64_t i = lo; i < std::min<int64_t>(lo + 4, n); ++i) {
                if (math_mode == MATH_LIBM) run_orbit<MATH_LIBM>(*run, i, *b, K, N, escape);
                else run_orbit<MATH_PORTABLE>(*run, i, *b, K, N, escape);
            }
        }
    };
    std::vector<std::thread> pool;
    for (int t = 1; t < nt; ++t) pool.emplace_back(worker);
    worker();
    for (auto& th : pool) th.join();
    return 0;
}

void oracle_sincos(int32_t mode, const double* x, double* s, double* c, int64_t n) {
    for (int64_t i = 0; i < n; ++i) {
        if (mode == MATH_LIBM) Math<MATH_LIBM>::sincos(x[i], s + i, c + i);
        else p_sincos(x[i], s + i, c + i);
    }
}

void oracle_log(int32_t mode, const double* x, double* y, int64_t n) {
    for (int64_t i = 0; i < n; ++i) y[i] = mode == MATH_LIBM ? std::log(x[i]) : p_log(x[i]);
}

void oracle_exp(int32_t mode, const double* x, double* y, int64_t n) {
    for (int64_t i = 0; i < n; ++i) y[i] = mode == MATH_LIBM ? std::exp(x[i]) : p_exp(x[i]);
}

void oracle_atan2(int32_t mode, const double* y, const double* x, double* a, int64_t n) {
    for (int64_t i = 0; i < n; ++i) a[i] = mode == MATH_LIBM ? std::atan2(y[i], x[i]) : p_atan2(y[i], x[i]);
}

void oracle_fused_product(const double* A, const double* B, double* C, int32_t m, int32_t p, int32_t nn) {
    fused_product(A, B, C, m, p, nn);
}

double oracle_safe_norm(const double* v, int32_t n) { return safe_norm(v, n); }

int32_t oracle_orthonormalize(int32_t alg, const double* W, int32_t d, int32_t k, double* Q, double* R,
                              int32_t* count, int32_t* status, int32_t* column) {
    const QRResult r = orthonormalize(alg, W, d, k, Q, R);
    *count = r.count; *status = r.status; *column = r.column;
    return 0;
}

double oracle_window_Gw(const double* R, int32_t k) { return window_Gw(R, k); }
double oracle_orth_loss(const double* Q, int32_t d, int32_t k) { return orth_loss(Q, d, k); }

void oracle_seeded_frame(uint64_t seed, int64_t orbit, int32_t d, int32_t k, double* W) {
    seeded_frame<MATH_PORTABLE>(seed, orbit, d, k, W);
}

// One Gauss-3 step of the Henon-Heiles flow: advances z (4) and writes the 4 x 4 tangent T.
int32_t oracle_gauss3_step(double* z, double h, int32_t maxiter, double tol, double* T) {
    Gauss3 g(maxiter, tol);
    g.step(z, h, T);
    return 0;
}

// One step of a table method on the Henon-Heiles flow: advances z (4) and writes the 4 x 4 tangent T.
int32_t oracle_split_step(double* z, double h, int32_t n_stages, const double* c, const double* d, double* T) {
    const SplitHH s{n_stages, c, d};
    s.step(z, h, T);
    return 0;
}

// The two-trajectory estimator on the CPU: one window [run.n0, run.n0 + steps) of n orbits (see the C ABI); with
// `grid`, the recorder's rows and failing grid indices as well.
int oracle_shadow(const cl_run* run, int64_t n, const double* x0, const double* u0, void* ends, double d0,
                  int32_t math_mode, int32_t threads, const int64_t* grid, int32_t n_grid, double* R, int64_t* fail) {
    const int64_t steps = run->steps > 0 ? run->steps : run->N - run->n0;
    if (run->tau <= 0 || steps % run->tau != 0 || run->n0 + steps > run->N) return CL_EINVAL;
    const int hw = static_cast<int>(std::max(1u, std::thread::hardware_concurrency()));
    const int nt = static_cast<int>(std::min<int64_t>(threads > 0 ? threads : hw, std::max<int64_t>(n, 1)));
    std::atomic<int64_t> next{0};
    auto worker = [&]() {
        for (;;) {
            const int64_t lo = next.fetch_add(16);
            if (lo >= n) return;
            for (int64_t i = lo; i < std::min<int64_t>(lo + 16, n); ++i) {
                if (math_mode == MATH_LIBM)
                    shadow_orbit<MATH_LIBM>(*run, i, x0, u0, static_cast<uint8_t*>(ends), d0, run->n0, steps, grid,
                                            n_grid, R, fail);
                else
                    shadow_orbit<MATH_PORTABLE>(*run, i, x0, u0, static_cast<uint8_t*>(ends), d0, run->n0, steps, grid,
                                                n_grid, R, fail);
            }
        }
    };
    std::vector<std::thread> pool;
    for (int t = 1; t < nt; ++t) pool.emplace_back(worker);
    worker();
    for (auto& th : pool) th.join();
    return 0;
}

// The recorder on the CPU: one window [run.n0, run.n0 + steps) of n orbits, buffers in place (see the C ABI).
int oracle_record(const cl_run* run, int64_t n, double* x, double* W, void* states, int8_t* code, int64_t* hstep,
                  const int64_t* grid, int32_t n_grid, double* R, int64_t* fail, int32_t math_mode, int32_t threads) {
    const int64_t steps = run->steps > 0 ? run->steps : run->N - run->n0;
    if (run->tau <= 0 || steps % run->tau != 0 || run->n0 + steps > run->N || run->n_frames != 1) return CL_EINVAL;
    const int hw = static_cast<int>(std::max(1u, std::thread::hardware_concurrency()));
    const int nt = static_cast<int>(std::min<int64_t>(threads > 0 ? threads : hw, std::max<int64_t>(n, 1)));
    std::atomic<int64_t> next{0};
    auto worker = [&]() {
        for (;;) {
            const int64_t lo = next.fetch_add(16);
            if (lo >= n) return;
            for (int64_t i = lo; i < std::min<int64_t>(lo + 16, n); ++i) {
                if (math_mode == MATH_LIBM)
                    rec_orbit<MATH_LIBM>(*run, i, x, W, static_cast<uint8_t*>(states), code, hstep, grid, n_grid, R, fail,
                                         run->n0, steps);
                else
                    rec_orbit<MATH_PORTABLE>(*run, i, x, W, static_cast<uint8_t*>(states), code, hstep, grid, n_grid, R,
                                             fail, run->n0, steps);
            }
        }
    };
    std::vector<std::thread> pool;
    for (int t = 1; t < nt; ++t) pool.emplace_back(worker);
    worker();
    for (auto& th : pool) th.join();
    return 0;
}

// The indicator recorder on the CPU: one window [run.n0, run.n0 + steps) of n orbits, buffers in place (see the
// C ABI's cl_b200_indicator_device); R has ncols(chain) + 3 + ns columns per row.
// pair != 0: the stream is PairMap(run->sys), x holds 2 s and W (2 d) x 2 entries per orbit.
int oracle_indicator(const cl_run* run, int32_t pair, int64_t n, int32_t ns, double* x, double* W, void* states,
                     int8_t* code, int64_t* hstep, const int64_t* grid, int32_t n_grid, double* R, int64_t* fail,
                     int32_t math_mode, int32_t threads) {
    const int64_t steps = run->steps > 0 ? run->steps : run->N - run->n0;
    if (run->tau <= 0 || steps % run->tau != 0 || run->n0 + steps > run->N || run->n_frames != 1 ||
        run->frames[0].k != 2 || ns < 0 || ns > (pair ? 2 : 1) * run->s)
        return CL_EINVAL;
    const int hw = static_cast<int>(std::max(1u, std::thread::hardware_concurrency()));
    const int nt = static_cast<int>(std::min<int64_t>(threads > 0 ? threads : hw, std::max<int64_t>(n, 1)));
    std::atomic<int64_t> next{0};
    auto worker = [&]() {
        for (;;) {
            const int64_t lo = next.fetch_add(16);
            if (lo >= n) return;
            for (int64_t i = lo; i < std::min<int64_t>(lo + 16, n); ++i) {
                if (math_mode == MATH_LIBM)
                    ind_orbit<MATH_LIBM>(*run, pair != 0, i, ns, x, W, static_cast<uint8_t*>(states), code, hstep,
                                         grid, n_grid, R, fail, run->n0, steps);
                else
                    ind_orbit<MATH_PORTABLE>(*run, pair != 0, i, ns, x, W, static_cast<uint8_t*>(states), code,
                                             hstep, grid, n_grid, R, fail, run->n0, steps);
            }
        }
    };
    std::vector<std::thread> pool;
    for (int t = 1; t < nt; ++t) pool.emplace_back(worker);
    worker();
    for (auto& th : pool) th.join();
    return 0;
}

// advance_ensemble (src/Integrators/ensemble.jl:1-45) on the CPU: `steps` steps of size sys->dt from every state
// of x0 (n x 4) into out, ok per orbit. A table method runs advance_n (stepper.jl:27-48: the kick weight held back
// while no drift follows, across the step boundary too); Gauss(3) runs advance_checked per step and stops at a
// failed step with the all-NaN state (gauss.jl:143-147, ensemble.jl:5-11).
int oracle_advance(const cl_system* sys, int64_t n, const double* x0, double* out, uint8_t* ok, int64_t steps,
                   int32_t threads) {
    if (sys->kind != CL_SYS_HH_SPLIT && sys->kind != CL_SYS_HH_GAUSS) return CL_EUNSUPPORTED;
    const int hw = static_cast<int>(std::max(1u, std::thread::hardware_concurrency()));
    const int nt = static_cast<int>(std::min<int64_t>(threads > 0 ? threads : hw, std::max<int64_t>(n, 1)));
    std::atomic<int64_t> next{0};
    auto orbit = [&](int64_t i) {
        double z[4];
        std::memcpy(z, x0 + 4 * i, sizeof z);
        uint8_t good = 1;
        const double dt = sys->dt;
        if (sys->kind == CL_SYS_HH_SPLIT && sys->corrector) {   // advance_n(::CorrectedMethod), stepper.jl:142-152
            const SplitHH m = SplitHH::of(*sys);
            for (int64_t s = 0; s < steps; ++s) m.forward(z, dt);
        } else if (sys->kind == CL_SYS_HH_SPLIT) {
            double pend = 0.0;
            for (int64_t s = 0; s < steps; ++s)
                for (int k = 0; k < sys->n_stages; ++k) {
                    const double ck = sys->stage_c[k];
                    if (ck != 0.0) {
                        if (pend != 0.0) { hh_kick(z, pend * dt); pend = 0.0; }
                        hh_drift(z, ck * dt);
                    }
                    pend = pend + sys->stage_d[k];
                }
            if (pend != 0.0) hh_kick(z, pend * dt);
        } else {
            const Gauss3 g(sys->gauss_maxiter, sys->gauss_tol);
            for (int64_t s = 0; s < steps; ++s) {
                double inc[4], Y[3][4];
                if (!g.core(z, dt, inc, Y)) {
                    for (double& v : z) v = std::numeric_limits<double>::quiet_NaN();
                    good = 0;
                    break;
                }
                for (int l = 0; l < 4; ++l) z[l] = z[l] + inc[l];
            }
        }
        std::memcpy(out + 4 * i, z, sizeof z);
        ok[i] = good;
    };
    auto worker = [&]() {
        for (;;) {
            const int64_t lo = next.fetch_add(16);
            if (lo >= n) return;
            for (int64_t i = lo; i < std::min<int64_t>(lo + 16, n); ++i) orbit(i);
        }
    };
    std::vector<std::thread> pool;
    for (int t = 1; t < nt; ++t) pool.emplace_back(worker);
    worker();
    for (auto& th : pool) th.join();
    return 0;
}

// The window kinds on the CPU: one window [run.n0, run.n0 + steps) of n orbits, buffers in place (see the C ABI's
// cl_b200_indicator_window_device).
int oracle_indicator_window(const cl_run* run, const cl_window* win, int64_t n, int32_t ns, double* x, void* states,
                            int8_t* code, int64_t* hstep, const int64_t* grid, int32_t n_grid, double* R,
                            int64_t* fail, int32_t math_mode, int32_t threads) {
    const int64_t steps = run->steps > 0 ? run->steps : run->N - run->n0;
    if (run->tau <= 0 || steps % run->tau != 0 || run->n0 + steps > run->N || ns < 0 || ns > run->s) return CL_EINVAL;
    const int hw = static_cast<int>(std::max(1u, std::thread::hardware_concurrency()));
    const int nt = static_cast<int>(std::min<int64_t>(threads > 0 ? threads : hw, std::max<int64_t>(n, 1)));
    std::atomic<int64_t> next{0};
    auto worker = [&]() {
        for (;;) {
            const int64_t lo = next.fetch_add(16);
            if (lo >= n) return;
            for (int64_t i = lo; i < std::min<int64_t>(lo + 16, n); ++i) {
                if (math_mode == MATH_LIBM)
                    win_orbit<MATH_LIBM>(*run, *win, i, ns, x, static_cast<uint8_t*>(states), code, hstep, grid, n_grid,
                                         R, fail, run->n0, steps);
                else
                    win_orbit<MATH_PORTABLE>(*run, *win, i, ns, x, static_cast<uint8_t*>(states), code, hstep, grid,
                                             n_grid, R, fail, run->n0, steps);
            }
        }
    };
    std::vector<std::thread> pool;
    for (int t = 1; t < nt; ++t) pool.emplace_back(worker);
    worker();
    for (auto& th : pool) th.join();
    return 0;
}

int32_t oracle_max_threads(void) { return static_cast<int32_t>(std::max(1u, std::thread::hardware_concurrency())); }

}  // extern "C"
