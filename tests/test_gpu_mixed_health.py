"""Health checks of the mixed precision's Gram-Schmidt frames against the Float64 run.

A Float32 frame applies QRSpectrum's checks with Float32's epsilon, as the reference does for a Float32 element type
(effective_eps(T), qr_spectrum.jl:54-73): the conditioning check of the Gram-Schmidt family fails once
G_w eps(Float32) >= 1/2 (G_w ~ 4.2e6), a window the Float64 run still passes. These tests state where the codes of the
two runs must agree and that every Float32 conditioning stop is one the Float64 record predicts."""
from __future__ import annotations

import numpy as np
import pytest

from chaos_b200 import MGS, FroeschleMap, QRSpectrum, WrappedStandardMap, propagate_frames, torus_state
from chaos_b200.propagate import FrameSpec
from helpers import identity_frames, same_bits, uniform_starts

pytestmark = pytest.mark.gpu

EPS32 = float(np.finfo(np.float32).eps)


def test_mixed_mgs_codes_agree_at_tau_1():
    """C1's frame (MGS, k = 2, tau = 1: one-step windows, G_w ~ 40): every orbit has the Float64 run's code and step."""
    n = 4096
    x0 = np.array([torus_state(v) for v in uniform_starts(n, 2, 1)])
    sysm = WrappedStandardMap(6.0)
    fr = [FrameSpec(2, (QRSpectrum(MGS()),), identity_frames(n, 2, 2))]
    a = propagate_frames(sysm, x0, 20000, fr, tau=1, finals=False, throw=False)[0]
    b = propagate_frames(sysm, x0, 20000, fr, tau=1, precision="mixed", finals=False, throw=False)[0]
    assert same_bits(a.x, b.x)
    assert np.array_equal(a.code, b.code) and np.array_equal(a.hstep, b.hstep)
    assert np.all(a.code == 0)


def test_mixed_mgs_conditioning_predicted():
    """Froeschle, MGS, k = 4, tau = 10 (chaotic windows of G_w up to ~1e9): where the Float64 record's G_max stays
    below 0.1 / eps(Float32) the Float32 frame completes like the Float64 one, point bit for bit; every Float32
    conditioning stop (code 3, value G_w eps >= 1/2) is on an orbit whose Float64 G_max reaches 0.25 / eps(Float32)
    (a Float32 G_w that ill-conditioned carries a relative error up to ~G_w eps(Float32)); no other code appears. On this
    workload most chaotic orbits stop (the Float64 G_max exceeds 1e7 on ~97 % of them), which is why the mixed
    headline reduces its QR frame by Householder, whose QRSpectrum has no conditioning check."""
    n, N = 4096, 10000
    x0 = uniform_starts(n, 4, 12)
    sysm = FroeschleMap(1.5, 1.5, 0.05)
    fr = [FrameSpec(4, (QRSpectrum(MGS()),), identity_frames(n, 4, 4))]
    a = propagate_frames(sysm, x0, N, fr, tau=10, finals=False, throw=False)[0]
    b = propagate_frames(sysm, x0, N, fr, tau=10, precision="mixed", finals=False, throw=False)[0]
    gmax = a.states["r0"]["G_max"]
    assert np.all(a.code == 0)
    well = gmax * EPS32 < 0.1
    assert well.sum() >= 20, well.sum()
    assert np.all(b.code[well] == 0) and np.all(b.hstep[well] == N)
    assert same_bits(a.x[well], b.x[well])
    cond = b.code == 3
    assert np.all(gmax[cond] * EPS32 >= 0.25), np.sort(gmax[cond] * EPS32)[:5]
    assert np.all(b.states["r0"]["value"][cond] >= 0.5)
    assert np.all((b.code == 0) | cond)
