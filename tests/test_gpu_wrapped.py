"""Parity of the torus forms of the coupled maps on the B200 with the oracle, bit for bit: WrappedFroeschleMap
(the C2 ensemble with its coordinates in [0, 2 pi)^4) under every compiled chain, fused frames included, and
WrappedStandardMapChain for N = 2..8 with open and ring boundaries; the mixed kernels against the plain one
(the orbit bit for bit, lambda_1 within 1e-3); count overflow reported as a non-finite state on the device too."""
from __future__ import annotations

import math

import numpy as np
import pytest

from chaos_b200 import (CGS, FLI, GALI, MEGNO, MGS, SALI, Benettin, GivensQR, HouseholderQR, QRSpectrum,
                        WrappedFroeschleMap, WrappedStandardMapChain, propagate_frames, torus_state)
from chaos_b200.propagate import FrameSpec
from helpers import haar_frames, identity_frames, same_bits, states_equal

pytestmark = pytest.mark.gpu

FRO = WrappedFroeschleMap(1.5, 1.5, 0.05)


def _compare(sysm, x0, N, frames, tau, oracle):
    dev = propagate_frames(sysm, x0, N, frames, tau=tau, finals=False, throw=False)
    ref = oracle.oracle_frames(sysm, x0, N, frames, tau=tau, math="portable")
    for f in range(len(frames)):
        assert same_bits(dev[f].x, ref[f]["x"]), f"x differs (frame {f})"
        assert np.array_equal(dev[f].code, ref[f]["code"]) and np.array_equal(dev[f].hstep, ref[f]["hstep"])
        assert same_bits(dev[f].W, ref[f]["W"]), f"W differs (frame {f})"
        assert states_equal(dev[f].states, ref[f]["states"]), f"states differ (frame {f})"
    return dev


def _torus_starts(sysm, n, seed, lo=-20.0, hi=20.0):
    z = np.random.default_rng(seed).uniform(lo, hi, (n, sysm.d))
    return np.array([torus_state(sysm, v) for v in z])


@pytest.mark.parametrize("k,chain", [(1, (Benettin(),)), (1, (QRSpectrum(CGS()),)), (1, (QRSpectrum(MGS()),)),
                                     (2, (QRSpectrum(MGS()),)), (2, (QRSpectrum(GivensQR()),)), (2, (SALI(),)),
                                     (2, (MEGNO(),)), (2, (FLI(),)),
                                     (2, (MEGNO(replace=False), FLI(replace=False), QRSpectrum(GivensQR()))),
                                     (2, (MEGNO(replace=False), SALI())), (4, (QRSpectrum(HouseholderQR()),)),
                                     (4, (QRSpectrum(MGS()),)), (4, (GALI(),)), (4, (GALI(), SALI()))], ids=repr)
def test_wrapped_froeschle(oracle, k, chain):
    n = 256
    x0 = _torus_starts(FRO, n, 41)
    _compare(FRO, x0, 2000, [FrameSpec(k, chain, haar_frames(n, 4, k, 42))], 10, oracle)


def test_wrapped_froeschle_fused_and_mixed(oracle):
    """The C2 frames (QRSpectrum(Householder) | GALI_4 + SALI) on one torus orbit; the mixed kernel keeps the orbit
    bit for bit and lambda_1 within 1e-3."""
    n = 512
    x0 = _torus_starts(FRO, n, 51, 0.0, 2 * math.pi)
    W0 = identity_frames(n, 4, 4)
    frames = [FrameSpec(4, (QRSpectrum(HouseholderQR()),), W0), FrameSpec(4, (GALI(), SALI()), W0)]
    dev = _compare(FRO, x0, 5000, frames, 10, oracle)
    mx = propagate_frames(FRO, x0, 5000, frames, tau=10, precision="mixed", finals=False, throw=False)
    assert same_bits(mx[0].x, dev[0].x)
    ok = (dev[0].code == 0) & (mx[0].code == 0)
    l64 = (dev[0].states["r0"]["sums"][:, 0, 0] + dev[0].states["r0"]["sums"][:, 0, 1]) / 5000
    lmx = (mx[0].states["r0"]["sums"][:, 0, 0] + mx[0].states["r0"]["sums"][:, 0, 1]) / 5000
    assert ok.mean() > 0.99 and np.max(np.abs(l64[ok] - lmx[ok])) <= 1e-3


@pytest.mark.parametrize("N_sites", range(2, 9))
@pytest.mark.parametrize("ring", [False, True])
def test_wrapped_chain(oracle, N_sites, ring):
    if ring and N_sites < 3:
        pytest.skip("a ring needs N >= 3")
    d = 2 * N_sites
    n = 128
    sysm = WrappedStandardMapChain(N_sites, 1.2, 0.05, boundary="ring" if ring else "open")
    x0 = _torus_starts(sysm, n, 60 + N_sites)
    k = min(d, 8)
    for chain in ((QRSpectrum(MGS()),), (QRSpectrum(HouseholderQR()),), (GALI(),)):
        _compare(sysm, x0, 500, [FrameSpec(k, chain, haar_frames(n, d, k, 70))], 5, oracle)
    for chain in ((QRSpectrum(MGS()),), (SALI(),), (MEGNO(),)):
        _compare(sysm, x0, 500, [FrameSpec(2, chain, haar_frames(n, d, 2, 71))], 5, oracle)
    _compare(sysm, x0, 500, [FrameSpec(1, (Benettin(),), haar_frames(n, d, 1, 72))], 5, oracle)
    fr = [FrameSpec(k, (QRSpectrum(MGS()),), haar_frames(n, d, k, 73))]
    a = propagate_frames(sysm, x0, 500, fr, tau=5, finals=False, throw=False)[0]
    b = propagate_frames(sysm, x0, 500, fr, tau=5, precision="mixed", finals=False, throw=False)[0]
    assert same_bits(a.x, b.x)
    ok = (a.code == 0) & (b.code == 0)
    la = (a.states["r0"]["sums"][:, 0, 0] + a.states["r0"]["sums"][:, 0, 1]) / 500
    lb = (b.states["r0"]["sums"][:, 0, 0] + b.states["r0"]["sums"][:, 0, 1]) / 500
    assert np.max(np.abs(la[ok] - lb[ok])) <= 1e-3


def test_count_overflow_on_the_device(oracle):
    lim = 2.0 ** 53
    x0 = np.array([[6.0, 0.0, 3.0, 0.0, lim - 1, 0.0, 0.0, 0.0], [6.0, 0.0, 3.0, 0.0, lim - 2, 0.0, 0.0, 0.0]])
    sysm = WrappedFroeschleMap(0.0, 0.0, 0.0)
    dev = _compare(sysm, x0, 1, [FrameSpec(2, (QRSpectrum(MGS()),), identity_frames(2, 4, 2))], 1, oracle)
    assert dev[0].code.tolist() == [1, 0]
    chain = WrappedStandardMapChain(2, 6.0, 0.0)
    x0 = np.array([[math.pi / 2, 0.0, 1.0, 0.0, 0.0, 0.0, lim - 1, 0.0],
                   [math.pi / 2, 0.0, 1.0, 0.0, 0.0, 0.0, lim - 2, 0.0]])
    dev = _compare(chain, x0, 1, [FrameSpec(2, (QRSpectrum(MGS()),), identity_frames(2, 4, 2))], 1, oracle)
    assert dev[0].code.tolist() == [1, 0]
