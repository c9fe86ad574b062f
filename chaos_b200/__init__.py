"""chaos_b200: the B200 (sm_100a) engine for Chaoslab's ensemble hot path.

`propagate(sys, x0, N; k, tau, seed, reducers)` of the Julia package Chaoslab (src/Tangent/propagate.jl:279-290),
running in the fused orbit kernels of libchaoslab_b200 (chaos_b200/csrc) behind the C ABI of
include/chaoslab_b200.h. This Python package is the host side of that boundary: the reference's systems and
reducers as parameter records, the argument checks, chunking, error and summary records.
"""
from .foundation import FALLBACK_REASONS, DeviceError, NumericalHealthError
from .diagnostics import eps_pair, eps_sum, spectrum_residuals, sum_threshold
from .propagate import (FrameSpec, PropagationResult, build_run, bytes_per_orbit, chunk_size, probe, propagate,
                        propagate_frames, propagate_orbit, release_cache)
from .reducers import (CGS, FLI, GALI, MEGNO, MGS, RGS, RLI, SALI, AugmentedQR, Benettin, GivensQR, HouseholderQR,
                       QRSpectrum)
from .advance import advance_ensemble
from .record import pair_frame, pair_start, record, record_indicator_pairs, record_indicators, record_shadow
from .shadow import propagate_shadow
from .systems import (ABA864, ABAH864, PEFRL, SABA, SABAC, SBAB, SBABC, CalvoSanzSerna4, CorrectedMethod, ForestRuth,
                      FroeschleMap, Gauss, HenonHeilesFlow, IntegratorMap, KahanLi, Leapfrog, LinearSymplecticMap,
                      McLachlan2, Ruth3, SofroniouSpaletta10, SplittingMethod, StandardMap, StandardMapChain,
                      SymplecticEuler, WrappedFroeschleMap, WrappedStandardMap, WrappedStandardMapChain, Yoshida, adjoint_method, coefficients, energy_start,
                      force_evaluations, is_palindromic, isolated_force_evaluations, lift, method_name, method_source,
                      nominal_order, random_energy_starts, section_interval, stage_count, suzuki_jump, table_digits,
                      torus_state, triple_jump, rotation_block, hyperbolic_block, block_diagonal, conjugated)

__all__ = [
    "propagate", "propagate_frames", "propagate_orbit", "propagate_shadow", "record", "record_indicators", "record_indicator_pairs", "pair_start", "pair_frame", "record_shadow", "advance_ensemble", "FrameSpec", "PropagationResult", "build_run", "bytes_per_orbit", "chunk_size",
    "probe", "release_cache", "eps_sum", "eps_pair", "sum_threshold", "spectrum_residuals", "NumericalHealthError", "DeviceError", "FALLBACK_REASONS",
    "QRSpectrum", "CGS", "MGS", "RGS", "HouseholderQR", "AugmentedQR", "GivensQR", "Benettin", "SALI", "GALI",
    "MEGNO", "FLI", "RLI",
    "StandardMap", "WrappedStandardMap", "FroeschleMap", "WrappedFroeschleMap", "StandardMapChain",
    "WrappedStandardMapChain", "rotation_block", "hyperbolic_block", "block_diagonal", "conjugated", "LinearSymplecticMap", "IntegratorMap",
    "Gauss", "SplittingMethod", "CorrectedMethod", "SymplecticEuler", "Leapfrog", "McLachlan2", "Ruth3", "ForestRuth",
    "triple_jump", "suzuki_jump", "PEFRL", "CalvoSanzSerna4", "Yoshida", "KahanLi", "SofroniouSpaletta10", "SABA",
    "SBAB", "SABAC", "SBABC", "ABA864", "ABAH864", "adjoint_method", "coefficients", "stage_count", "nominal_order",
    "is_palindromic", "table_digits", "force_evaluations", "isolated_force_evaluations", "method_name",
    "method_source", "HenonHeilesFlow", "torus_state", "lift", "energy_start", "random_energy_starts", "section_interval",
]
