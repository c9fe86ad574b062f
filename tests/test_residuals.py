"""The residual records of a spectrum (src/Diagnostics/residuals.jl:13-32): eps_sum, eps_pair and sum_threshold,
their definitions, the oracle's spectra against them, and on the GPU the configurations' full-size runs: the
standard map K = 6 (4096 orbits x 1e5 steps, MGS, tau = 1), whose two exponents sum to 0 within 1e-12, and the
coupled maps (65536 x 1e5, Householder, tau = 10), whose four exponents pair."""
from types import SimpleNamespace

import numpy as np
import pytest

from chaos_b200 import (FroeschleMap, HouseholderQR, MGS, QRSpectrum, StandardMap, WrappedStandardMap, eps_pair,
                        eps_sum, sum_threshold)
from chaos_b200.diagnostics import EPS32, spectrum_residuals
from chaos_b200.foundation import EPS
from chaos_b200.propagate import FrameSpec, propagate_frames
from helpers import identity_frames, uniform_starts


def test_definitions():
    """eps_sum = |sum|, eps_pair = max_i |l_i + l_(M+1-i)| in estimator order (no sorting), and the threshold
    tol eps(T) (G_max / tau + M_max) with the reference's default multiplier 16."""
    lam = np.array([0.7, 0.2, -0.25, -0.65])
    assert eps_sum(lam) == abs(((0.7 + 0.2) + -0.25) + -0.65)
    assert eps_pair(lam) == max(abs(0.7 - 0.65), abs(0.2 - 0.25))
    assert eps_pair(np.array([0.7, -0.25, 0.2, -0.65])) == max(abs(0.7 - 0.65), abs(-0.25 + 0.2))   # not sorted
    assert eps_pair(np.array([1.0, -1.0])) == 0.0
    with pytest.raises(ValueError):
        eps_pair(np.array([1.0]))
    assert sum_threshold(16, "Float64", 40.0, 10, 7.0) == 16 * EPS * (40.0 / 10 + 7.0)
    assert sum_threshold(16, "Float32", 40.0, 10, 7.0) == 16 * EPS32 * (40.0 / 10 + 7.0)
    assert StandardMap(6.0).tangent_bound() == 7.0


def _oracle_result(oracle, sysm, x0, N, k, alg, tau):
    fr = [FrameSpec(k, (QRSpectrum(alg),), identity_frames(len(x0), sysm.d, k))]
    ref = oracle.oracle_frames(sysm, x0, N, fr, tau=tau, math="portable")[0]
    return SimpleNamespace(reducers=(QRSpectrum(alg),), states=ref["states"], code=ref["code"])


def test_oracle_standard_map_sum(oracle):
    """The oracle's two exponents of the standard map K = 6 (tau = 1, MGS) sum to zero within 1e-12 and within
    sum_threshold (README.md:19-22: lambda = +-1.13486)."""
    x0 = uniform_starts(64, 2, seed=1)
    r = _oracle_result(oracle, StandardMap(6.0), x0, 4000, 2, MGS(), 1)
    res = spectrum_residuals(r, tau=1, system=StandardMap(6.0))
    assert np.all(r.code == 0)
    assert np.max(res["eps_sum"]) <= 1e-12 and np.all(res["sum_ok"])
    assert np.all(res["eps_pair"] == res["eps_sum"])   # k = 2: the pair is the sum
    assert 0.9 < np.median(res["lam"][:, 0]) < 1.4


def test_oracle_froeschle_sum(oracle):
    """The coupled maps' four exponents (Householder, tau = 10) sum to zero within sum_threshold."""
    x0 = uniform_starts(32, 4, seed=2)
    sysm = FroeschleMap(1.5, 1.5, 0.05)
    r = _oracle_result(oracle, sysm, x0, 3000, 4, HouseholderQR(), 10)
    res = spectrum_residuals(r, tau=10, system=sysm)
    assert np.all(r.code == 0) and np.all(res["sum_ok"])


@pytest.mark.gpu
def test_standard_map_full_sum():
    """The standard map K = 6 at its full size (4096 orbits, (x, p) uniform on the torus, N = 1e5, k = 2, W0 = I,
    tau = 1, QRSpectrum(MGS)) on the torus map: every orbit's exponents sum to 0 within 1e-12 and within
    sum_threshold, in the Float64 kernel; the mixed kernel (Float32 frame) within the Float32 threshold."""
    n, N = 4096, 100_000
    sysm = WrappedStandardMap(6.0)
    x0 = np.array([sysm.torus_state(zi) for zi in uniform_starts(n, 2, seed=1)])
    fr = [FrameSpec(2, (QRSpectrum(MGS()),), identity_frames(n, 2, 2))]
    r = propagate_frames(sysm, x0, N, fr, tau=1, finals=False, throw=False)[0]
    assert np.all(r.code == 0)
    res = r.spectrum_residuals(sysm)
    assert np.max(res["eps_sum"]) <= 1e-12 and np.all(res["sum_ok"])
    assert 1.0 < np.median(res["lam"][:, 0]) < 1.3
    rm = propagate_frames(sysm, x0, N, fr, tau=1, precision="mixed", finals=False, throw=False)[0]
    ok = rm.code == 0
    assert ok.mean() > 0.99
    assert np.all(rm.spectrum_residuals(sysm)["sum_ok"][ok])


@pytest.mark.gpu
def test_froeschle_full_pairing():
    """The coupled maps at full size (65536 orbits uniform in [0, 2 pi)^4, N = 1e5, k = 4, W0 = I, tau = 10,
    Householder): every sum within sum_threshold, and the exponents pair (l1 + l4, l2 + l3) within 1e-3."""
    n, N = 65536, 100_000
    x0 = uniform_starts(n, 4, seed=1)
    sysm = FroeschleMap(1.5, 1.5, 0.05)
    fr = [FrameSpec(4, (QRSpectrum(HouseholderQR()),), identity_frames(n, 4, 4))]
    r = propagate_frames(sysm, x0, N, fr, tau=10, finals=False, throw=False)[0]
    ok = r.code == 0
    assert ok.mean() > 0.999
    res = r.spectrum_residuals(sysm)
    assert np.all(res["sum_ok"][ok])
    assert np.max(res["eps_pair"][ok]) <= 1e-3
