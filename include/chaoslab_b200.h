/*
 * chaoslab_b200.h -- C ABI of libchaoslab_b200, the B200 (sm_100a) engine for Chaoslab's ensemble hot path
 * `propagate(sys, x0s, N; k, tau, seed, reducers)`.
 *
 * The reference reaches its device through Julia hooks, not a C ABI: `Tangent._run_chunk!` launches the
 * KernelAbstractions kernel `_orbit_kernel!` (src/Tangent/propagate.jl:32-50, launch at :105, synchronize :106),
 * and ext/ChaoslabCUDAExt.jl:16-93 fills the device hooks of src/Foundation/Foundation.jl:84-104. A Julia
 * package extension binds the entry points below with `ccall` in place of that launch. The ABI carries only plain
 * pointers, sizes and POD structs.
 *
 * Layouts (all host buffers are owned by the caller; no pointer is kept after a call returns):
 *  - x0, x   : n_orbits x s doubles, orbit-major (Julia `Vector{SVector{s,Float64}}`).
 *  - W0, W   : n_orbits x (d*k) doubles per frame, each matrix column-major (Julia `Vector{SMatrix{d,k,Float64}}`).
 *  - states  : n_orbits x cl_b200_state_bytes(run, f) bytes per frame, the isbits layout of the Julia tuple of
 *              reducer states (QRState, BenettinState, SALIState, GALIState, MEGNOState, FLIState with T = Float64),
 *              so `reducer_final` / `reducer_error` run unchanged on the host.
 *  - code    : n_orbits int8 per frame (STATUS_OK 0, STATE 1, W 2, REDUCER 3; src/Tangent/orbit.jl:1).
 *  - hstep   : n_orbits int64 per frame, the global step of the failing handoff, else the last step reached.
 *
 * Frames: one call integrates each orbit once and carries up to CL_MAX_FRAMES tangent frames along it, each with
 * its own k and reducer chain. A frame behaves as a separate reference `propagate` run on the same orbit and W0
 * (its own status, failing step, W and states); the orbit stops only when every frame has stopped. One frame is
 * exactly the reference call.
 *
 * Return codes: 0 success; negative values map one to one onto the reference's FALLBACK_REASONS indices
 * (src/Foundation/Foundation.jl:71-75): -2 no functional device (reason 2), -3 kernel not built for this system /
 * chain / precision (reason 3), -4 device out of memory (reason 4), -9 device lost or a bounded device wait
 * timed out (reason 9); -1 is an invalid argument (the reference throws ArgumentError before any work).
 * Per-orbit numerical failures are not call errors: they come back in code / hstep / states. After a non-zero
 * return the contents of the output arrays (x, W, states, code, hstep and the in/out arrays among them) are
 * unspecified: a failure that surfaces at the final synchronisation can come after their copies began.
 */
#ifndef CHAOSLAB_B200_H
#define CHAOSLAB_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#if defined(__GNUC__)
#define CL_API __attribute__((visibility("default")))
#else
#define CL_API
#endif

#define CL_B200_ABI_VERSION 3
#define CL_MAX_FRAMES 3
#define CL_MAX_REDUCERS 4
#define CL_MAX_DIM 16
#define CL_MAX_K 8
#define CL_MAX_STAGES 128
#define CL_MAX_WINDOWS 4
#define CL_MAX_OBSERVABLES 8

/* Systems (src/Systems): the fixed menu the compiled kernels cover. */
enum cl_system_kind {
    CL_SYS_STANDARD = 1,         /* StandardMap(K), d = s = 2                       standard_map.jl:8-44        */
    CL_SYS_WRAPPED_STANDARD = 2, /* WrappedStandardMap(K), d = 2, s = 4              wrapped_standard_map.jl:12-57 */
    CL_SYS_FROESCHLE = 3,        /* FroeschleMap(nu, kappa, mu), d = s = 4           froeschle_map.jl:9-58       */
    CL_SYS_CHAIN = 4,            /* StandardMapChain(N, K, eps), d = s = 2N          standard_map_chain.jl:11-31 */
    CL_SYS_LINEAR = 5,           /* LinearSymplecticMap(A), d = s                    linear_symplectic.jl:1-40   */
    CL_SYS_HH_GAUSS = 6,         /* IntegratorMap(Gauss(Float64, 3; tol), HenonHeilesFlow(), dt), d = s = 4
                                    integrator_map.jl:12-23, gauss.jl:49-192, flow_models.jl:101-103        */
    CL_SYS_HH_SPLIT = 7,         /* IntegratorMap(SplittingMethod(c, d), HenonHeilesFlow(), dt), d = s = 4: a table
                                    method (drift c_i dt, then kick d_i dt), forward with merged kicks, tangent the
                                    product of the stage Jacobians; stepper.jl:27-48,108-118, flow_core.jl:59-72  */
    CL_SYS_WRAPPED_FROESCHLE = 8, /* WrappedFroeschleMap(nu, kappa, mu), d = 4, s = 8: (x1, x2, p1, p2) in [0, 2pi)
                                    and four exact winding counts; froeschle_map.jl:60-126                     */
    CL_SYS_WRAPPED_CHAIN = 9     /* WrappedStandardMapChain(N, K, eps), d = 2N, s = 4N: (q, p) in [0, 2pi) and 2N
                                    exact winding counts; wrapped_standard_map_chain.jl:1-154                  */
};

/* Reducers (src/Lyapunov, src/Indicators). */
enum cl_reducer_kind {
    CL_RED_QR = 1,       /* QRSpectrum(alg; orthogonality_tol)   qr_spectrum.jl:14-96 */
    CL_RED_BENETTIN = 2, /* Benettin()                          benettin.jl:11-53    */
    CL_RED_SALI = 3,     /* SALI()                              sali.jl:14-68        */
    CL_RED_GALI = 4,     /* GALI()                              gali.jl:17-201       */
    CL_RED_MEGNO = 5,    /* MEGNO(; replace)                    megno.jl:29-113      */
    CL_RED_FLI = 6,      /* FLI(; replace)                      fli.jl:26-96         */
    CL_RED_RLI = 7       /* RLI(; replace), on a pair stream    rli.jl:24-114        */
};

/* Orthonormalizers of QRSpectrum (orthonormalize.jl:5-12, householder.jl:5-10). */
enum cl_qr_alg {
    CL_QR_CGS = 1,
    CL_QR_MGS = 2,
    CL_QR_RGS = 3,
    CL_QR_HOUSEHOLDER = 4,
    CL_QR_AUGMENTED = 5,
    CL_QR_GIVENS = 6
};

/* Arithmetic of the tangent frames. The orbit, the Gauss-Legendre solve and the log sums are Float64 in both. */
enum cl_precision {
    CL_PREC_FP64 = 0, /* plain kernel: the reference's Float64 algorithm, operation for operation           */
    CL_PREC_MIXED = 1, /* tangent frames and their QR / norms in Float32, log sums Float64 (Neumaier)        */
    CL_PREC_MIXED_IND64 = 2 /* Float32 Lyapunov frames (QRSpectrum), Float64 indicator frames (GALI, SALI), the
                             * orbit Float64; compiled for the coupled-maps pair QRSpectrum(Householder) k = 4 |
                             * GALI + SALI k = 4 (cl_split_frames.cu)                                            */
};

enum cl_status {
    CL_OK = 0,
    CL_EINVAL = -1,
    CL_ENODEVICE = -2,
    CL_EUNSUPPORTED = -3,
    CL_ENOMEM = -4,
    CL_EDEVICE_LOST = -9
};

typedef struct cl_system {
    int32_t kind;          /* enum cl_system_kind                                                       */
    int32_t n_sites;       /* CL_SYS_CHAIN, CL_SYS_WRAPPED_CHAIN: N in 2..8                             */
    int32_t ring;          /* the chains: 1 for boundary = :ring (N >= 3), 0 for :open                  */
    int32_t gauss_maxiter; /* CL_SYS_HH_GAUSS: fixed-point iteration cap (reference default 50)         */
    double K;              /* standard maps and chain                                                   */
    double eps;            /* chain coupling                                                            */
    double nu, kappa, mu;  /* Froeschle parameters                                                      */
    double gauss_tol;      /* absolute stage tolerance; NaN = the reference's 8 eps max(1, |Y|) bound   */
    double dt;             /* IntegratorMap step tau of the flow                                        */
    double A[CL_MAX_DIM * CL_MAX_DIM]; /* CL_SYS_LINEAR: d x d matrix, column-major                     */
    int32_t n_stages;      /* CL_SYS_HH_SPLIT: stages k of the table, 1..CL_MAX_STAGES                          */
    int32_t corrector;     /* CL_SYS_HH_SPLIT: 1 for CorrectedMethod(table, c) (SABAC / SBABC): the corrector
                              kick p += kappa grad|grad V|^2 before and after every step, kappa = dt^3 c / 2 with
                              c in `eps` (stepper.jl:131-160, tables_near.jl:113-128); else 0                   */
    double stage_c[CL_MAX_STAGES]; /* CL_SYS_HH_SPLIT: drift weights c_1..c_k (splitting.jl:16-21)      */
    double stage_d[CL_MAX_STAGES]; /* CL_SYS_HH_SPLIT: kick weights d_1..d_k                            */
} cl_system;

typedef struct cl_reducer {
    int32_t kind;             /* enum cl_reducer_kind                                   */
    int32_t alg;              /* CL_RED_QR: enum cl_qr_alg                              */
    int32_t replace;          /* CL_RED_MEGNO / CL_RED_FLI: the `replace` keyword (0/1) */
    int32_t pad;
    double orthogonality_tol; /* CL_RED_QR: reference default 8.0                       */
} cl_reducer;

typedef struct cl_frame {
    int32_t k;          /* deviation vectors, 1 <= k <= d */
    int32_t n_reducers; /* 0..CL_MAX_REDUCERS             */
    cl_reducer reducers[CL_MAX_REDUCERS];
} cl_frame;

typedef struct cl_run {
    int32_t abi_version; /* CL_B200_ABI_VERSION                                                          */
    int32_t d;           /* dimension(sys)                                                               */
    int32_t s;           /* state length (>= d; 4 for the wrapped standard map's winding counts)         */
    int32_t tau;         /* handoff interval                                                             */
    int64_t N;           /* steps of the whole run, a positive multiple of tau                           */
    int64_t n0;          /* first global step of this launch: 0 starts fresh, > 0 continues carried state */
    int64_t steps;       /* steps in this launch (a multiple of tau); 0 means N - n0                     */
    int32_t n_frames;    /* 1..CL_MAX_FRAMES                                                             */
    int32_t precision;   /* enum cl_precision                                                            */
    uint64_t seed;       /* seed of the Haar frames drawn when a frame's W0 is NULL                      */
    int64_t orbit_base;  /* id of orbit 0 of this call minus one (orbit ids are 1-based, as in Julia)    */
    cl_system sys;
    cl_frame frames[CL_MAX_FRAMES];
} cl_run;

/* Buffers of one call. For n0 == 0, x0 / W0 are read and x / W / states / code / hstep written; W0[f] may be
 * NULL (seeded Haar frame). For n0 > 0, x / W / states / code are read as the carried state (x0, W0 unused), an
 * orbit whose code is not 0 is not advanced, and everything is written back in place. */
typedef struct cl_buffers {
    const double* x0;
    double* x;
    const double* W0[CL_MAX_FRAMES];
    double* W[CL_MAX_FRAMES];
    void* states[CL_MAX_FRAMES];
    int8_t* code[CL_MAX_FRAMES];
    int64_t* hstep[CL_MAX_FRAMES];
} cl_buffers;

/* What a call ran, for the run's provenance (propagate.jl:260-264 records backend, device, launch_steps,
 * launches_per_chunk; these are the device-side counterparts). */
typedef struct cl_prov {
    char device[96];      /* device name                                    */
    char variant[160];    /* compiled kernel instance that ran              */
    int64_t launch_steps; /* steps per launch                               */
    int64_t launches;     /* kernel launches of the orbit kernel            */
    double gpu_ms;        /* device time of the orbit kernel launches       */
    int32_t block;        /* threads per block                              */
    int32_t grid;         /* blocks per launch                              */
    int32_t regs;         /* registers per thread of the instance           */
    int32_t orbits_per_block;
} cl_prov;

/* Backend probe: the (loadable, functional, device, compiles, gpu_faster) record of Foundation.probe
 * (src/Foundation/Foundation.jl:92-93, ext/ChaoslabCUDAExt.jl:87-91). */
typedef struct cl_probe {
    int32_t loadable;
    int32_t functional;
    int32_t compiles;
    int32_t sm;          /* compute capability x 10, e.g. 100 */
    int64_t free_bytes;  /* Foundation.free_memory             */
    int64_t total_bytes;
    int32_t sm_count;
    int32_t pad;
    char device[96];
} cl_probe;

/* propagate one chunk, host buffers: copies in, runs the orbit kernel in launches of at most run->steps steps,
 * copies out. Replaces `_run_chunk!` (src/Tangent/propagate.jl:92-119) for a device chunk. */
CL_API int cl_b200_propagate(const cl_run* run, int64_t n_orbits, const cl_buffers* host, cl_prov* prov);

/* The same on device buffers already resident in GPU memory, enqueued on `stream` (a cudaStream_t; NULL is the
 * legacy default stream). `soa` = 1 takes x / W as structure-of-arrays (component-major: element c of orbit i at
 * c * n_orbits + i) for coalesced loads; 0 takes the orbit-major host layout. States and code / hstep are always
 * orbit-major. Returns after the launch is enqueued. */
CL_API int cl_b200_propagate_device(const cl_run* run, int64_t n_orbits, const cl_buffers* dev, int32_t soa, void* stream);

/* Autotune the register budget of the instance that covers `run`: times each compiled variant (1, 2, 3 or 4
 * resident blocks of 128 threads per SM) over `sample_steps` steps of the n_orbits
 * orbits on the device buffers (whose contents are overwritten), remembers the fastest for this run's instance and
 * tau in the process, and writes it to *minb_out. Later propagate calls of the same instance use it. No reference
 * counterpart. */
CL_API int cl_b200_tune(const cl_run* run, int64_t n_orbits, const cl_buffers* dev, int32_t soa, int64_t sample_steps,
                        void* stream, int32_t* minb_out);
/* The compiled variants of the instance that covers `run` as a bit set (bit v - 1: variant v), 0 if none covers it;
 * and pinning one of them for this run's instance and tau, as cl_b200_tune would (variant 0 clears the pin, the next
 * public call then tunes again). CL_EINVAL for a variant the instance does not have. No reference counterpart. */
CL_API int32_t cl_b200_variants(const cl_run* run);
CL_API int cl_b200_set_variant(const cl_run* run, int32_t variant);

/* 0 when a compiled kernel instance covers `run`, else CL_EINVAL (ill-formed run, message in cl_b200_last_error)
 * or CL_EUNSUPPORTED (well-formed, but not in the compiled menu: the caller falls back with reason 3). */
CL_API int cl_b200_check(const cl_run* run);

/* Bytes per orbit of frame f's reducer-state tuple in the Julia isbits layout (0 for an empty chain). */
CL_API int64_t cl_b200_state_bytes(const cl_run* run, int32_t frame);

/* Fill `out`; returns 0 when a B200-class device is functional. */
CL_API int cl_b200_probe(cl_probe* out);

/* Copy the message of the last failed call on this thread; returns its length. */
CL_API int cl_b200_last_error(char* buf, size_t len);

/* Library version string. */
CL_API const char* cl_b200_version(void);

/* Number of orbit-kernel launches since the library was loaded (a device-launch counter for audits). */
CL_API int64_t cl_b200_launch_count(void);

/* The host-buffer entry points take their device buffers from a stream-ordered pool per device that the library
 * owns and that keeps its memory between calls (a call of the same sizes as an earlier one allocates nothing from
 * the driver). This returns the memory the pools keep to the driver; a later call grows them again. The
 * counterpart of CUDA.jl's `CUDA.reclaim()` for the memory pool the reference's device runs allocate from. */
CL_API int cl_b200_release_cache(void);

/* ---- Batched uneven ensembles ------------------------------------------------------------------------------------
 * One class = orbits of one system kind and dimension with one frame and chain; every orbit may carry its own map
 * parameter K (K[i]), its own length N[i] (a multiple of tau) and an escape stop: at the first handoff where
 * max_j |p_j| > escape the orbit stops with code 4 (STATUS_ESCAPED) and its records are those of the reference call
 * `propagate_orbit(sys(K[i]), x0[i], W0[i], N', tau, reducers)` with N' that handoff (src/Tangent/orbit.jl:85-99).
 * The reference has one N, one system and no escape per call, so an ensemble is the set of such calls. Orbits are
 * taken from a device work queue in `order` (longest first balances the load) by persistent kernels, one per class,
 * all classes concurrently. Buffers are orbit-major (frame 0 of each class's cl_buffers). */
typedef struct cl_ensemble_class {
    cl_run run;            /* system, d, s, tau, one frame, precision; run.N is the length when N is NULL      */
    int64_t n_orbits;
    const int64_t* order;  /* queue: n_orbits orbit indices (NULL: 0..n-1)                                     */
    const double* K;       /* per-orbit K (NULL: run.sys.K); standard maps and chains                          */
    const int64_t* N;      /* per-orbit lengths, multiples of tau, each <= run.N (NULL: run.N)                 */
    double escape;         /* momentum bound of the escape stop; <= 0 disables it                              */
    int32_t minb;          /* kernel variant: register cap as blocks per SM (1, 2 or 4); 0 = tuned/default     */
    int32_t unroll;        /* kernel variant: tau loop unrolled (tau itself, when tau is 5, 10 or 20) or 1; 0 = tuned/default */
    cl_buffers buf;        /* frame 0 only                                                                      */
    int32_t lanes;         /* kernel variant: lanes per orbit, 1 (one orbit per thread) or, for lattices of
                              2, 4 or 8 sites reduced by QRSpectrum(HouseholderQR) with k a multiple of the sites and
                              an explicit W0, the number of sites (the sites and the frame's columns spread over
                              that many lanes); 0 = tuned/default                                               */
    int32_t reserved;      /* 0                                                                                 */
} cl_ensemble_class;

/* Run the classes on device buffers, enqueued on `stream`; the queue heads are allocated and freed in stream
 * order (cudaMallocAsync). No reference counterpart (see above). */
CL_API int cl_b200_ensemble_device(const cl_ensemble_class* classes, int32_t n_classes, void* stream);

/* The same without allocating anything, for callers that cannot allocate GPU memory while they call in (a host
 * whose own allocator owns the device heap, a plugin host that forbids allocation calls, a latency-bound loop).
 * No counterpart in the reference. The classes run one after another on `stream`; their queue heads live in a
 * fixed array inside the library, CL_NOALLOC_MAX_CLASSES heads (512 bytes) held on every GPU that loads the
 * library until exit, and more classes than that are rejected with CL_EINVAL. Every call looks the array's device
 * address up in the current context (no allocation; allowed during stream capture, so a call can be captured into
 * a CUDA graph of memset and kernel nodes), clears the heads it uses on `stream`, and a call whose classes are
 * rejected enqueues nothing; calls that overlap on the GPU race on the shared array. */
#define CL_NOALLOC_MAX_CLASSES 64
CL_API int cl_b200_ensemble_device_noalloc(const cl_ensemble_class* classes, int32_t n_classes, void* stream);

/* The same on host buffers: copies in, runs, copies out (synchronous). */
CL_API int cl_b200_ensemble(const cl_ensemble_class* classes, int32_t n_classes, cl_prov* prov);

/* Autotune one class on its device buffers: times every kernel variant (register cap, tau unrolling, lanes per
 * orbit) on a sample of the queue and writes the fastest (minb, unroll, lanes) into the class. The sample is
 * `sample_orbits` queue slots at an even stride (all of them when <= 0 or >= n_orbits) with every length scaled by
 * sample_steps / run.N, so the longest orbit keeps its share of the work. The buffers' contents are overwritten. */
CL_API int cl_b200_ensemble_tune(cl_ensemble_class* cls, int64_t sample_orbits, int64_t sample_steps, void* stream);

/* Capture the classes' launches (queue resets included) into one CUDA graph on device buffers; launching the
 * graph replays the whole ensemble. The graph owns its queue heads until destroyed. */
CL_API int cl_b200_ensemble_graph_create(const cl_ensemble_class* classes, int32_t n_classes, void** graph);
CL_API int cl_b200_ensemble_graph_launch(void* graph, void* stream);
CL_API int cl_b200_ensemble_graph_destroy(void* graph);

/* ---- The two-trajectory estimator (src/Lyapunov/two_trajectory.jl:40-96, separation.jl) ---------------------------
 * Per orbit a shadow started at displaced(x0, d0 u0) (u0 a unit vector of the d tangent coordinates), both orbits
 * advanced by `forward`; every tau steps the separation d is measured, log(d / d_prev) is added to a Neumaier sum and
 * the shadow is put back at distance d0 along the separation. `ends` holds one record per orbit in the isbits layout
 * of the reference's ShadowEnd{s, Float64}: x[s], y[s], sum (s, c), dprev, code (Int8 in an 8-byte slot: 0 ok,
 * 1 non-finite state, 2 separation zero or non-finite, 3 realised separation outside [d0/2, 2 d0]), step (Int64),
 * value; X2 = (sum.s + sum.c) / N. run.n0 == 0 starts the shadows (u0 NULL: the first column of the seeded frame of
 * the run's seed and orbit_base + i + 1), a later window continues from `ends` and leaves failed orbits untouched.
 * run.frames are not used. Replaces the launch loop of `_shadow_chunk!` (two_trajectory.jl:123-143). */
CL_API int64_t cl_b200_shadow_bytes(int32_t s);
/* One launch window [run.n0, run.n0 + run.steps) (run.steps 0: to run.N) on device buffers, enqueued on `stream`. */
CL_API int cl_b200_shadow_device(const cl_run* run, int64_t n, const double* x0, const double* u0, void* ends,
                                 double d0, void* stream);
/* The same from run.n0 to run.N on host buffers, in windows of run.steps steps (synchronous). */
CL_API int cl_b200_shadow(const cl_run* run, int64_t n, const double* x0, const double* u0, void* ends, double d0,
                          cl_prov* prov);
/* The recorder's two-trajectory method (src/Experiments/run_device.jl:80-100): segments between the grid steps
 * (increasing multiples of run.tau); at each grid step g of the window, row g of R[col, g, orbit] (8 + s columns,
 * zeroed by the caller) gets X2 so far (sum / step) in column 1 and the reference state in columns 9..8+s; a failure
 * stores the 1-based grid index whose segment holds it in fail[orbit] (zeroed by the caller). Replaces
 * `_shadow_record_kernel!` launches. Device buffers, enqueued on `stream`; the host form runs every window. */
CL_API int cl_b200_shadow_record_device(const cl_run* run, int64_t n, const double* x0, const double* u0, void* ends,
                                        double d0, const int64_t* grid, int32_t n_grid, double* R, int64_t* fail,
                                        void* stream);
CL_API int cl_b200_shadow_record(const cl_run* run, int64_t n, const double* x0, const double* u0, void* ends,
                                 double d0, const int64_t* grid, int32_t n_grid, double* R, int64_t* fail,
                                 cl_prov* prov);

/* ---- The study recorder (src/Experiments/run_device.jl:43-78, run_record.jl:24-40) ------------------------------
 * One launch window [run.n0, run.n0 + run.steps) of the variational methods with grid records: the orbit body runs
 * segment by segment between the grid steps (`grid`, increasing multiples of run.tau) and at every grid step inside
 * the window writes one row of R[col, g, orbit] (Julia column-major, Float64), cl_b200_record_columns(run) =
 * k + 7 + s columns: lambda (k), det_max, symp_max, orth_max, running max of eps_sum, running max of eps_pair,
 * G_max, M_max, the state (s); det / symp / M are the running maxima of the non-raising monitor (|det M - 1|,
 * max|M' Omega M - Omega|, max|M|, M the tangent at the handoff point). For k = 1 the sum and pair columns are left
 * as they are. A failure stores the 1-based grid index whose segment holds it in fail[orbit] and stops the orbit.
 * x, W, states (the estimator's state then MonState{Float64}: cl_b200_record_state_bytes(run) bytes per orbit),
 * code and hstep are carried in place; x and W hold x0 and W0 before the first window, R and fail must be zero.
 * Systems: StandardMap, WrappedStandardMap, 2 x 2 LinearSymplecticMap; run.frames[0]: Benettin with k = 1 or
 * QRSpectrum(CGS, MGS, RGS, Householder, augmented) with k = 2; Float64. Replaces `_record_kernel!` launches. */
CL_API int32_t cl_b200_record_columns(const cl_run* run);
CL_API int64_t cl_b200_record_state_bytes(const cl_run* run);
CL_API int cl_b200_record_device(const cl_run* run, int64_t n, double* x, double* W, void* states, int8_t* code,
                                 int64_t* hstep, const int64_t* grid, int32_t n_grid, double* R, int64_t* fail,
                                 void* stream);
/* The same from run.n0 to run.N on host buffers, in windows of run.steps steps (synchronous). */
CL_API int cl_b200_record(const cl_run* run, int64_t n, double* x, double* W, void* states, int8_t* code,
                          int64_t* hstep, const int64_t* grid, int32_t n_grid, double* R, int64_t* fail, cl_prov* prov);

/* ---- The indicator recorder, window kinds (src/Experiments/run_indicator_device.jl:62-91) --------------------------
 * The phase-advance and Birkhoff kinds: the orbit of the base map (run.sys, run.d = 2, frames[0].k = 1, no reducers)
 * advanced one handoff at a time with the deviation column reset to (1, 0) at each handoff, the non-raising monitor
 * and one reader reducer: WeightedPhaseAdvance (src/Indicators/naff_reducer.jl:122-243) or WeightedBirkhoff
 * (wbirkhoff_reducer.jl:18-110), with the Birkhoff weight exp(-1 / (t^p (1 - t)^p)) at the mirrored index. At every
 * grid step one row of R[col, g, orbit] of 3 + ns columns: det_max, symp_max, M_max, x[0 .. ns-1]. states per orbit:
 * MonState{Float64} (24 bytes) then the reader's isbits state (cl_b200_window_state_bytes: WPAState{Float64, H},
 * 64 H + 32 bytes; WBState{Float64, H, K}, 16 + H (16 + 40 K) bytes), carried in place; the tables are the
 * reader's reducer_final on the host. fail: the 1-based grid index of the failing handoff's segment. */
enum cl_window_kind { CL_WIN_PHASE_ADVANCE = 1, CL_WIN_BIRKHOFF = 2 };
enum cl_observable_kind {
    CL_OBS_PLANAR = 1,       /* PlanarObservable(a, b): z = x[a] + i x[b]                naff_reducer.jl:96-101   */
    CL_OBS_LIFTED_ANGLE = 2, /* LiftedAngleObservable(a, b): (x[a], count x[b]; b = 0 none) naff_reducer.jl:103-117 */
    CL_OBS_COS = 3,          /* CosObservable(a, b): cos(b x[a])                          wbirkhoff.jl:12-23      */
    CL_OBS_SIN = 4,          /* SinObservable(a, b): sin(b x[a])                          wbirkhoff.jl:25-36      */
    CL_OBS_LIFTED = 5,       /* LiftedObservable(a, b): x[a] + 2 pi x[b]                  wbirkhoff.jl:38-49      */
    CL_OBS_COORDINATE = 6    /* IndCoordinate(a): x[a]                     src/Experiments/run_indicator_chain.jl:20-23 */
};
typedef struct cl_window {
    int32_t kind;            /* enum cl_window_kind                                                       */
    int32_t n_windows;       /* H, 1..CL_MAX_WINDOWS                                                      */
    int32_t n_observables;   /* K: 1 for the phase advance, 1..CL_MAX_OBSERVABLES for Birkhoff            */
    int32_t birkhoff_order;  /* p, 1..4                                                                   */
    int64_t window[CL_MAX_WINDOWS];       /* the horizons N_h, each >= 16                                 */
    int32_t obs_kind[CL_MAX_OBSERVABLES]; /* enum cl_observable_kind                                      */
    int32_t obs_a[CL_MAX_OBSERVABLES];    /* 1-based coordinate index                                     */
    int32_t obs_b[CL_MAX_OBSERVABLES];    /* second index (1-based, 0 = none) or the integer frequency    */
} cl_window;
CL_API int64_t cl_b200_window_state_bytes(const cl_window* win);
CL_API int cl_b200_indicator_window_device(const cl_run* run, const cl_window* win, int64_t n, int32_t ns, double* x,
                                           void* states, int8_t* code, int64_t* hstep, const int64_t* grid,
                                           int32_t n_grid, double* R, int64_t* fail, void* stream);
CL_API int cl_b200_indicator_window(const cl_run* run, const cl_window* win, int64_t n, int32_t ns, double* x,
                                    void* states, int8_t* code, int64_t* hstep, const int64_t* grid, int32_t n_grid,
                                    double* R, int64_t* fail, cl_prov* prov);

/* ---- advance_ensemble (src/Integrators/ensemble.jl:13-45) ---------------------------------------------------------
 * `steps` steps of size sys->dt of the integrator of an IntegratorMap system (CL_SYS_HH_SPLIT: a table method,
 * advanced by advance_n with the pending kick carried across step boundaries, stepper.jl:27-48; CL_SYS_HH_GAUSS:
 * Gauss(3), advance_checked per step, a failed step leaving the all-NaN state and ok = 0) on the Henon-Heiles flow,
 * from every state of x0 (n x 4 doubles, orbit-major, 32-byte aligned on the device) into out, ok one byte per
 * orbit. No tangent. Replaces `_ensemble_kernel!` launches; the result does not depend on the chunking. */
CL_API int cl_b200_advance_ensemble_device(const cl_system* sys, int64_t n, const double* x0, double* out,
                                           uint8_t* ok, int64_t steps, void* stream);
/* The same on host buffers, `chunk` orbits per launch (<= 0: all), synchronous. */
CL_API int cl_b200_advance_ensemble(const cl_system* sys, int64_t n, const double* x0, double* out, uint8_t* ok,
                                    int64_t steps, int64_t chunk, cl_prov* prov);

/* ---- The indicator recorder, tangent kind (src/Experiments/run_indicator_device.jl:13-60) ---------------------------
 * One launch window of a chain of indicator members on a k = 2 frame (run.frames[0]: SALI, MEGNO, FLI in one of the
 * compiled orders, every member but the last non-replacing, the last replacing) followed by the non-raising monitor.
 * At every grid step inside the window one row of R[col, g, orbit] (column-major, Float64) of
 * cl_b200_indicator_columns(run, ns) columns: the members' columns in chain order (SALI: sali, L; FLI: fli, fli1;
 * MEGNO: Y, Ybar, Ybar20 of column 1, then of column 2; run_indicator_record.jl:40-56), then det_max, symp_max,
 * M_max of the monitor, then x[0 .. ns-1]. fail[orbit] = the 1-based grid index whose segment holds the failure.
 * states = the members' states (cl_b200_state_bytes layout) then MonState{Float64} (24 bytes):
 * cl_b200_indicator_state_bytes(run) per orbit. Systems: StandardMap, WrappedStandardMap, 2 x 2 LinearSymplecticMap;
 * Float64. Replaces `_ind_series_kernel!` launches. cl_b200_indicator_columns is -1 for a chain outside the menu. */
CL_API int32_t cl_b200_indicator_columns(const cl_run* run, int32_t ns);
CL_API int64_t cl_b200_indicator_state_bytes(const cl_run* run);
CL_API int cl_b200_indicator_device(const cl_run* run, int64_t n, int32_t ns, double* x, double* W, void* states,
                                    int8_t* code, int64_t* hstep, const int64_t* grid, int32_t n_grid, double* R,
                                    int64_t* fail, void* stream);
/* The same from run.n0 to run.N on host buffers, in windows of run.steps steps (synchronous). */
CL_API int cl_b200_indicator(const cl_run* run, int64_t n, int32_t ns, double* x, double* W, void* states,
                             int8_t* code, int64_t* hstep, const int64_t* grid, int32_t n_grid, double* R,
                             int64_t* fail, cl_prov* prov);
/* The pair kind: the same body on PairMap(run.sys) (src/Systems/pair.jl:9-68) -- run.sys, run.d and run.s describe
 * the base map; z holds the pair state (state A; state B), 2 run.s doubles per orbit, and W the (2 run.d) x 2 block
 * frame, column-major; the chain's members are RLI and MEGNO (RLI1; RLI0, MEGNO1; MEGNO0, RLI1: the reference's pair
 * specs), RLI's columns DL, RLI (rli.jl:98-101); the monitor reads orbit A. ns <= 2 run.s. Replaces the pair kind's
 * `_ind_series_kernel!` launches. */
CL_API int32_t cl_b200_indicator_pair_columns(const cl_run* run, int32_t ns);
CL_API int cl_b200_indicator_pair_device(const cl_run* run, int64_t n, int32_t ns, double* z, double* W,
                                         void* states, int8_t* code, int64_t* hstep, const int64_t* grid,
                                         int32_t n_grid, double* R, int64_t* fail, void* stream);
CL_API int cl_b200_indicator_pair(const cl_run* run, int64_t n, int32_t ns, double* z, double* W, void* states,
                                  int8_t* code, int64_t* hstep, const int64_t* grid, int32_t n_grid, double* R,
                                  int64_t* fail, cl_prov* prov);

/* ---- The learned screen's kernels (no reference counterpart: the reference has no learned component) ---------------
 * All enqueue on `stream` and take device pointers. BF16 matrices are row-major with 16-byte aligned rows. */

/* C[M x N] = A[M x K] . B[N x K]^T on the tcgen05 tensor cores (BF16 operands, FP32 accumulator in tensor memory),
 * + bias[N] (NULL: none), epilogue 0 none / 1 GELU (tanh form, (x / 2)(1 + tanh u), u = sqrt(2/pi)
 * (x + 0.044715 x^3), tanh by the special-function unit); C32 (FP32) and/or Cbf16 written with row stride ldc;
 * pre (FP32, NULL: none) receives the value before the epilogue; accumulate adds the old C32. */
CL_API int cl_b200_gemm_bf16(const void* A, int32_t lda, const void* B, int32_t ldb, int32_t M, int32_t N, int32_t K,
                             const float* bias, int32_t epilogue, float* C32, void* Cbf16, int32_t ldc, float* pre,
                             int32_t accumulate, void* stream);
/* Packs a row-major BF16 matrix (rows x cols, row stride ld elements) into tiles of tile_rows (a multiple of 8) x 64
 * columns in the canonical K-major layout the tensor cores read, zero padded to whole tiles: tile (rt, kb) is
 * contiguous at byte (rt * ceil(cols / 64) + kb) * tile_rows * 128. dst holds ceil(rows / tile_rows) * tile_rows *
 * ceil(cols / 64) * 64 elements, 16-byte aligned. The fused forward pass reads its weights in this layout (tile_rows =
 * the layer's output rows: 256, 256, 256, 16). */
CL_API int cl_b200_mlp_pack_kmajor(const void* src, int32_t rows, int32_t cols, int32_t ld, int32_t tile_rows,
                                   void* dst, void* stream);
/* The screen network's inference pass, 64 -> 256 -> 256 -> 256 (GELU) -> 16 (linear), in one persistent kernel:
 * X (B x 64 BF16, contiguous), Wp1..Wp4 the packed weights (256 x 64, 256 x 256, 256 x 256, 16 x 256), b1..b4 the
 * biases (FP32), out (B x 16 FP32). Bit for bit the per-layer cl_b200_gemm_bf16 chain. max_ctas > 0 caps the grid
 * (default: one CTA per SM). Pointers 16-byte aligned. */
CL_API int cl_b200_mlp_forward_fused(const void* X, int32_t B, const void* Wp1, const void* Wp2, const void* Wp3,
                                     const void* Wp4, const float* b1, const float* b2, const float* b3,
                                     const float* b4, float* out, int32_t max_ctas, void* stream);
/* 0, or CL_EDEVICE_LOST after a bounded wait on an MMA or copy barrier (GEMM or fused pass) gave up. */
CL_API int cl_b200_mlp_status(void);
CL_API int cl_b200_transpose_bf16(const void* src, int32_t rows, int32_t cols, int32_t lds, void* dst, int32_t ldd,
                                  void* stream);
/* dH = dY * GELU'(pre), to BF16 (dHb) and / or FP32 (dH32). */
CL_API int cl_b200_gelu_backward(const float* dY, const float* pre, int64_t n, void* dHb, float* dH32, void* stream);
/* out[j] = sum_i X[i, j] (bias gradients). */
CL_API int cl_b200_col_sum(const float* X, int32_t rows, int32_t cols, int32_t ld, float* out, void* stream);
/* Per-row loss BCE(logit = column 0, label) + w_reg (column 1 - target)^2 and the mean-loss gradient dL/dlogits. */
CL_API int cl_b200_head_loss(const float* logits, int32_t B, int32_t ld, const float* label, const float* target,
                             float w_reg, float* grad, void* gradb, float* row_loss, void* stream);
/* Adam on FP32 weights (step t >= 1), refreshing their BF16 copy wb and its transpose wbt (rows x cols) if given. */
CL_API int cl_b200_adam(float* w, const float* g, float* m, float* v, int64_t n, float lr, float b1, float b2, float eps,
                        int32_t t, void* wb, void* wbt, int32_t rows, int32_t cols, void* stream);
CL_API int cl_b200_to_bf16(const float* x, int64_t n, void* y, void* stream);
/* Screening features of window `window` (ending at global step n) from the reducer states of the chain
 * (MEGNO(replace = false), SALI()) on a k = 2 frame: 3 per window, 4 more after the last; 64 per orbit. */
CL_API int cl_b200_screen_features(const void* states, int64_t n_orbits, int64_t n, int32_t window, int32_t windows,
                                   float* f32, void* fbf16, void* stream);

/* The compiled menu: number of kernel instances, and the key of instance i (NULL outside 0..size-1). A key reads
 * "s<system kind>d<d>p<precision>|k<k>:<reducer>,...|..." with reducers QR<alg>, BEN, SALI, GALI, MEGNO<replace>,
 * FLI<replace>, one "|"-terminated group per frame. No reference counterpart (Julia compiles on demand). */
CL_API int32_t cl_b200_menu_size(void);
CL_API const char* cl_b200_menu_key(int32_t i);

#ifdef __cplusplus
}
#endif

#endif /* CHAOSLAB_B200_H */
