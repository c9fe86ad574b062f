"""ctypes mirror of include/chaoslab_b200.h (the C ABI of libchaoslab_b200).

The structs here are byte-for-byte the ones in the header; `tests/test_abi.py` checks their sizes and offsets
against the compiled library.
"""
from __future__ import annotations

import ctypes as C

ABI_VERSION = 3
MAX_FRAMES = 3
MAX_REDUCERS = 4
MAX_STAGES = 128
MAX_DIM = 16
MAX_K = 8
NOALLOC_MAX_CLASSES = 64
MAX_WINDOWS = 4
MAX_OBSERVABLES = 8

# enum cl_system_kind
SYS_STANDARD, SYS_WRAPPED_STANDARD, SYS_FROESCHLE, SYS_CHAIN, SYS_LINEAR, SYS_HH_GAUSS, SYS_HH_SPLIT = 1, 2, 3, 4, 5, 6, 7
SYS_WRAPPED_FROESCHLE, SYS_WRAPPED_CHAIN = 8, 9
# enum cl_reducer_kind
RED_QR, RED_BENETTIN, RED_SALI, RED_GALI, RED_MEGNO, RED_FLI, RED_RLI = 1, 2, 3, 4, 5, 6, 7
# enum cl_qr_alg
QR_CGS, QR_MGS, QR_RGS, QR_HOUSEHOLDER, QR_AUGMENTED, QR_GIVENS = 1, 2, 3, 4, 5, 6
# enum cl_precision
PREC_FP64, PREC_MIXED, PREC_MIXED_IND64 = 0, 1, 2
# enum cl_window_kind, enum cl_observable_kind
WIN_PHASE_ADVANCE, WIN_BIRKHOFF = 1, 2
OBS_PLANAR, OBS_LIFTED_ANGLE, OBS_COS, OBS_SIN, OBS_LIFTED, OBS_COORDINATE = 1, 2, 3, 4, 5, 6
# enum cl_status
OK, EINVAL, ENODEVICE, EUNSUPPORTED, ENOMEM, EDEVICE_LOST = 0, -1, -2, -3, -4, -9


class cl_system(C.Structure):
    _fields_ = [
        ("kind", C.c_int32),
        ("n_sites", C.c_int32),
        ("ring", C.c_int32),
        ("gauss_maxiter", C.c_int32),
        ("K", C.c_double),
        ("eps", C.c_double),
        ("nu", C.c_double),
        ("kappa", C.c_double),
        ("mu", C.c_double),
        ("gauss_tol", C.c_double),
        ("dt", C.c_double),
        ("A", C.c_double * (MAX_DIM * MAX_DIM)),
        ("n_stages", C.c_int32),
        ("corrector", C.c_int32),
        ("stage_c", C.c_double * MAX_STAGES),
        ("stage_d", C.c_double * MAX_STAGES),
    ]


class cl_reducer(C.Structure):
    _fields_ = [
        ("kind", C.c_int32),
        ("alg", C.c_int32),
        ("replace", C.c_int32),
        ("pad", C.c_int32),
        ("orthogonality_tol", C.c_double),
    ]


class cl_frame(C.Structure):
    _fields_ = [
        ("k", C.c_int32),
        ("n_reducers", C.c_int32),
        ("reducers", cl_reducer * MAX_REDUCERS),
    ]


class cl_run(C.Structure):
    _fields_ = [
        ("abi_version", C.c_int32),
        ("d", C.c_int32),
        ("s", C.c_int32),
        ("tau", C.c_int32),
        ("N", C.c_int64),
        ("n0", C.c_int64),
        ("steps", C.c_int64),
        ("n_frames", C.c_int32),
        ("precision", C.c_int32),
        ("seed", C.c_uint64),
        ("orbit_base", C.c_int64),
        ("sys", cl_system),
        ("frames", cl_frame * MAX_FRAMES),
    ]


class cl_buffers(C.Structure):
    _fields_ = [
        ("x0", C.c_void_p),
        ("x", C.c_void_p),
        ("W0", C.c_void_p * MAX_FRAMES),
        ("W", C.c_void_p * MAX_FRAMES),
        ("states", C.c_void_p * MAX_FRAMES),
        ("code", C.c_void_p * MAX_FRAMES),
        ("hstep", C.c_void_p * MAX_FRAMES),
    ]


class cl_window(C.Structure):
    _fields_ = [("kind", C.c_int32), ("n_windows", C.c_int32), ("n_observables", C.c_int32),
                ("birkhoff_order", C.c_int32), ("window", C.c_int64 * MAX_WINDOWS),
                ("obs_kind", C.c_int32 * MAX_OBSERVABLES), ("obs_a", C.c_int32 * MAX_OBSERVABLES),
                ("obs_b", C.c_int32 * MAX_OBSERVABLES)]


class cl_prov(C.Structure):
    _fields_ = [
        ("device", C.c_char * 96),
        ("variant", C.c_char * 160),
        ("launch_steps", C.c_int64),
        ("launches", C.c_int64),
        ("gpu_ms", C.c_double),
        ("block", C.c_int32),
        ("grid", C.c_int32),
        ("regs", C.c_int32),
        ("orbits_per_block", C.c_int32),
    ]


class cl_probe(C.Structure):
    _fields_ = [
        ("loadable", C.c_int32),
        ("functional", C.c_int32),
        ("compiles", C.c_int32),
        ("sm", C.c_int32),
        ("free_bytes", C.c_int64),
        ("total_bytes", C.c_int64),
        ("sm_count", C.c_int32),
        ("pad", C.c_int32),
        ("device", C.c_char * 96),
    ]


class cl_ensemble_class(C.Structure):
    _fields_ = [
        ("run", cl_run),
        ("n_orbits", C.c_int64),
        ("order", C.c_void_p),
        ("K", C.c_void_p),
        ("N", C.c_void_p),
        ("escape", C.c_double),
        ("minb", C.c_int32),
        ("unroll", C.c_int32),
        ("buf", cl_buffers),
        ("lanes", C.c_int32),
        ("reserved", C.c_int32),
    ]


def state_bytes(kind: int, k: int) -> int:
    """Bytes of one reducer state in the Julia isbits layout (T = Float64)."""
    return {RED_QR: 16 * k + 72, RED_BENETTIN: 48, RED_SALI: 72, RED_GALI: 24 * k + 32,
            RED_MEGNO: 200, RED_FLI: 96, RED_RLI: 88}[kind]


def frame_state_bytes(frame: cl_frame) -> int:
    return sum(state_bytes(frame.reducers[r].kind, frame.k) for r in range(frame.n_reducers))


def declare(lib: C.CDLL) -> C.CDLL:
    """Set the argument and result types of every entry point of libchaoslab_b200."""
    P = C.POINTER
    lib.cl_b200_propagate.argtypes = [P(cl_run), C.c_int64, P(cl_buffers), P(cl_prov)]
    lib.cl_b200_propagate.restype = C.c_int
    lib.cl_b200_propagate_device.argtypes = [P(cl_run), C.c_int64, P(cl_buffers), C.c_int32, C.c_void_p]
    lib.cl_b200_propagate_device.restype = C.c_int
    lib.cl_b200_tune.argtypes = [P(cl_run), C.c_int64, P(cl_buffers), C.c_int32, C.c_int64, C.c_void_p,
                                 P(C.c_int32)]
    lib.cl_b200_tune.restype = C.c_int
    lib.cl_b200_check.argtypes = [P(cl_run)]
    lib.cl_b200_check.restype = C.c_int
    lib.cl_b200_state_bytes.argtypes = [P(cl_run), C.c_int32]
    lib.cl_b200_state_bytes.restype = C.c_int64
    lib.cl_b200_probe.argtypes = [P(cl_probe)]
    lib.cl_b200_probe.restype = C.c_int
    lib.cl_b200_last_error.argtypes = [C.c_char_p, C.c_size_t]
    lib.cl_b200_last_error.restype = C.c_int
    lib.cl_b200_version.argtypes = []
    lib.cl_b200_version.restype = C.c_char_p
    lib.cl_b200_launch_count.argtypes = []
    lib.cl_b200_launch_count.restype = C.c_int64
    lib.cl_b200_release_cache.argtypes = []
    lib.cl_b200_release_cache.restype = C.c_int
    lib.cl_b200_ensemble_device.argtypes = [P(cl_ensemble_class), C.c_int32, C.c_void_p]
    lib.cl_b200_ensemble_device.restype = C.c_int
    lib.cl_b200_ensemble_device_noalloc.argtypes = [P(cl_ensemble_class), C.c_int32, C.c_void_p]
    lib.cl_b200_ensemble_device_noalloc.restype = C.c_int
    lib.cl_b200_ensemble.argtypes = [P(cl_ensemble_class), C.c_int32, P(cl_prov)]
    lib.cl_b200_ensemble.restype = C.c_int
    lib.cl_b200_ensemble_tune.argtypes = [P(cl_ensemble_class), C.c_int64, C.c_int64, C.c_void_p]
    lib.cl_b200_shadow_bytes.argtypes = [C.c_int32]
    lib.cl_b200_shadow_bytes.restype = C.c_int64
    lib.cl_b200_shadow_device.argtypes = [P(cl_run), C.c_int64, C.c_void_p, C.c_void_p, C.c_void_p, C.c_double,
                                          C.c_void_p]
    lib.cl_b200_shadow_device.restype = C.c_int
    lib.cl_b200_shadow.argtypes = [P(cl_run), C.c_int64, P(C.c_double), P(C.c_double), C.c_void_p, C.c_double,
                                   P(cl_prov)]
    lib.cl_b200_shadow.restype = C.c_int
    lib.cl_b200_record_columns.argtypes = [P(cl_run)]
    lib.cl_b200_record_columns.restype = C.c_int32
    lib.cl_b200_record_state_bytes.argtypes = [P(cl_run)]
    lib.cl_b200_record_state_bytes.restype = C.c_int64
    lib.cl_b200_record_device.argtypes = [P(cl_run), C.c_int64, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                          C.c_void_p, C.c_void_p, C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p]
    lib.cl_b200_record_device.restype = C.c_int
    lib.cl_b200_record.argtypes = [P(cl_run), C.c_int64, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                   C.c_void_p, C.c_int32, C.c_void_p, C.c_void_p, P(cl_prov)]
    lib.cl_b200_record.restype = C.c_int
    lib.cl_b200_shadow_record_device.argtypes = [P(cl_run), C.c_int64, C.c_void_p, C.c_void_p, C.c_void_p, C.c_double,
                                                 C.c_void_p, C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p]
    lib.cl_b200_shadow_record_device.restype = C.c_int
    lib.cl_b200_shadow_record.argtypes = [P(cl_run), C.c_int64, C.c_void_p, C.c_void_p, C.c_void_p, C.c_double,
                                          C.c_void_p, C.c_int32, C.c_void_p, C.c_void_p, P(cl_prov)]
    lib.cl_b200_shadow_record.restype = C.c_int
    lib.cl_b200_advance_ensemble_device.argtypes = [P(cl_system), C.c_int64, C.c_void_p, C.c_void_p, C.c_void_p,
                                                    C.c_int64, C.c_void_p]
    lib.cl_b200_advance_ensemble_device.restype = C.c_int
    lib.cl_b200_advance_ensemble.argtypes = [P(cl_system), C.c_int64, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int64,
                                             C.c_int64, P(cl_prov)]
    lib.cl_b200_advance_ensemble.restype = C.c_int
    lib.cl_b200_variants.argtypes = [P(cl_run)]
    lib.cl_b200_variants.restype = C.c_int32
    lib.cl_b200_set_variant.argtypes = [P(cl_run), C.c_int32]
    lib.cl_b200_set_variant.restype = C.c_int
    lib.cl_b200_indicator_columns.argtypes = [P(cl_run), C.c_int32]
    lib.cl_b200_indicator_columns.restype = C.c_int32
    lib.cl_b200_indicator_state_bytes.argtypes = [P(cl_run)]
    lib.cl_b200_indicator_state_bytes.restype = C.c_int64
    lib.cl_b200_indicator_device.argtypes = [P(cl_run), C.c_int64, C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p,
                                             C.c_void_p, C.c_void_p, C.c_void_p, C.c_int32, C.c_void_p, C.c_void_p,
                                             C.c_void_p]
    lib.cl_b200_indicator_device.restype = C.c_int
    lib.cl_b200_indicator.argtypes = [P(cl_run), C.c_int64, C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p,
                                      C.c_void_p, C.c_void_p, C.c_void_p, C.c_int32, C.c_void_p, C.c_void_p,
                                      P(cl_prov)]
    lib.cl_b200_indicator.restype = C.c_int
    lib.cl_b200_indicator_pair_columns.argtypes = [P(cl_run), C.c_int32]
    lib.cl_b200_indicator_pair_columns.restype = C.c_int32
    lib.cl_b200_indicator_pair_device.argtypes = lib.cl_b200_indicator_device.argtypes
    lib.cl_b200_indicator_pair_device.restype = C.c_int
    lib.cl_b200_indicator_pair.argtypes = lib.cl_b200_indicator.argtypes
    lib.cl_b200_indicator_pair.restype = C.c_int
    lib.cl_b200_window_state_bytes.argtypes = [P(cl_window)]
    lib.cl_b200_window_state_bytes.restype = C.c_int64
    lib.cl_b200_indicator_window_device.argtypes = [P(cl_run), P(cl_window), C.c_int64, C.c_int32, C.c_void_p,
                                                    C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int32,
                                                    C.c_void_p, C.c_void_p, C.c_void_p]
    lib.cl_b200_indicator_window_device.restype = C.c_int
    lib.cl_b200_indicator_window.argtypes = [P(cl_run), P(cl_window), C.c_int64, C.c_int32, C.c_void_p, C.c_void_p,
                                             C.c_void_p, C.c_void_p, C.c_void_p, C.c_int32, C.c_void_p, C.c_void_p,
                                             P(cl_prov)]
    lib.cl_b200_indicator_window.restype = C.c_int
    lib.cl_b200_ensemble_tune.restype = C.c_int
    lib.cl_b200_ensemble_graph_create.argtypes = [P(cl_ensemble_class), C.c_int32, P(C.c_void_p)]
    lib.cl_b200_ensemble_graph_create.restype = C.c_int
    lib.cl_b200_ensemble_graph_launch.argtypes = [C.c_void_p, C.c_void_p]
    lib.cl_b200_ensemble_graph_launch.restype = C.c_int
    lib.cl_b200_ensemble_graph_destroy.argtypes = [C.c_void_p]
    lib.cl_b200_ensemble_graph_destroy.restype = C.c_int
    lib.cl_b200_menu_size.argtypes = []
    lib.cl_b200_menu_size.restype = C.c_int32
    lib.cl_b200_menu_key.argtypes = [C.c_int32]
    lib.cl_b200_menu_key.restype = C.c_char_p
    return lib


# Every symbol include/chaoslab_b200.h declares (checked by the CPU tests against the built library).
EXPORTS = ("cl_b200_propagate", "cl_b200_propagate_device", "cl_b200_check", "cl_b200_state_bytes",
           "cl_b200_probe", "cl_b200_last_error", "cl_b200_version", "cl_b200_launch_count", "cl_b200_release_cache",
           "cl_b200_menu_size", "cl_b200_menu_key", "cl_b200_ensemble_device", "cl_b200_ensemble",
           "cl_b200_ensemble_tune", "cl_b200_ensemble_graph_create", "cl_b200_ensemble_graph_launch",
           "cl_b200_ensemble_graph_destroy", "cl_b200_ensemble_device_noalloc", "cl_b200_tune",
           "cl_b200_gemm_bf16", "cl_b200_mlp_pack_kmajor", "cl_b200_mlp_forward_fused", "cl_b200_mlp_status", "cl_b200_transpose_bf16", "cl_b200_gelu_backward",
           "cl_b200_col_sum", "cl_b200_head_loss", "cl_b200_adam", "cl_b200_to_bf16", "cl_b200_screen_features",
           "cl_b200_shadow_bytes", "cl_b200_shadow_device", "cl_b200_shadow", "cl_b200_record_columns",
           "cl_b200_record_state_bytes", "cl_b200_record_device", "cl_b200_record",
           "cl_b200_shadow_record_device", "cl_b200_shadow_record", "cl_b200_indicator_columns",
           "cl_b200_indicator_state_bytes", "cl_b200_indicator_device", "cl_b200_indicator",
           "cl_b200_advance_ensemble_device", "cl_b200_advance_ensemble", "cl_b200_indicator_pair_columns",
           "cl_b200_indicator_pair_device", "cl_b200_indicator_pair", "cl_b200_window_state_bytes",
           "cl_b200_indicator_window_device", "cl_b200_indicator_window", "cl_b200_variants",
           "cl_b200_set_variant")
