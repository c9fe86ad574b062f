"""`propagate` on coupled standard-map lattices with d >= 8 runs one orbit per group of lanes (cl_coop_orbit.cuh: the
sites over the lanes, neighbours by warp shuffles, QRSpectrum(HouseholderQR) column-parallel at the handoffs, every
other reducer chain on the group's first lane over the frame in shared memory). It must give the one-thread
kernel's records bit for bit -- point, frame, reducer states in the Julia layout, status and step -- in Float64 (where
the one-thread kernel is the oracle's arithmetic, checked in test_gpu_parity.py::test_chain, which now runs the
cooperative form by default) and in the mixed precision, across lattice sizes with and without idle lanes (d = 10,
12, 14 use groups of 8 lanes), open and ring lattices, seeded frames, relaunched windows and failures."""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

from chaos_b200 import GALI, MEGNO, MGS, SALI, Benettin, HouseholderQR, QRSpectrum, StandardMapChain, propagate_frames
from chaos_b200._lib import lib
from chaos_b200.propagate import FrameSpec, build_run
from helpers import haar_frames, same_bits, states_equal, uniform_starts

pytestmark = pytest.mark.gpu

V_ONE, V_COOP = 1, 8


def _run(sysm, x0, N, fr, tau, precision, variant, **kw):
    r = build_run(sysm, N, tau, [fr], precision, 7)
    L = lib()
    assert L.cl_b200_variants(C.byref(r)) & (1 << (V_COOP - 1)), "no cooperative variant for this instance"
    assert L.cl_b200_set_variant(C.byref(r), variant) == 0
    try:
        return propagate_frames(sysm, x0, N, [fr], tau=tau, seed=7, precision=precision, finals=False, throw=False,
                                **kw)[0]
    finally:
        L.cl_b200_set_variant(C.byref(r), 0)


def _same(a, b):
    assert same_bits(a.x, b.x)
    assert np.array_equal(a.code, b.code) and np.array_equal(a.hstep, b.hstep)
    assert same_bits(a.W, b.W)
    assert states_equal(a.states, b.states)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("sites,ring", [(4, False), (4, True), (5, True), (7, False), (8, False), (8, True)])
def test_coop_equals_one_thread(sites, ring, precision):
    d = 2 * sites
    n = 96
    sysm = StandardMapChain(sites, 1.1, 0.05, boundary="ring" if ring else "open")
    x0 = uniform_starts(n, d, 200 + sites)
    k = min(d, 8)
    cases = [(k, (QRSpectrum(HouseholderQR()),)), (k, (QRSpectrum(MGS()),)), (k, (GALI(),)),
             (2, (QRSpectrum(MGS()),)), (2, (SALI(),)), (2, (MEGNO(),))]
    if precision == "fp64":
        cases.append((1, (Benettin(),)))
    for kk, chain in cases:
        fr = FrameSpec(kk, chain, haar_frames(n, d, kk, 300 + sites))
        a = _run(sysm, x0, 600, fr, 5, precision, V_ONE)
        b = _run(sysm, x0, 600, fr, 5, precision, V_COOP)
        _same(a, b)


def test_coop_seeded_and_relaunch():
    """Seeded Haar frames drawn by the group's first lane, and a run split into launches of 70 steps: bit for bit
    the one-thread kernel's one-launch run."""
    sysm = StandardMapChain(8, 1.4, 0.05)
    n, d = 200, 16
    x0 = uniform_starts(n, d, 9)
    for chain in ((QRSpectrum(HouseholderQR()),), (QRSpectrum(MGS()),), (GALI(),)):
        fr = FrameSpec(8, chain, None)
        a = _run(sysm, x0, 700, fr, 10, "fp64", V_ONE)
        b = _run(sysm, x0, 700, fr, 10, "fp64", V_COOP, launch_steps=70)
        _same(a, b)


def test_coop_failures():
    """A non-finite start (state), an overflowing frame (deviation matrix) and a zero column (QR pivot, GALI norm)
    report the one-thread kernel's code, step and reducer record."""
    sysm = StandardMapChain(6, 1.2, 0.05, boundary="ring")
    n, d = 64, 12
    x0 = uniform_starts(n, d, 3)
    x0[3, 5] = np.nan
    for chain in ((QRSpectrum(HouseholderQR()),), (QRSpectrum(MGS()),), (GALI(),)):
        W0 = haar_frames(n, d, 8, 4)
        W0[5, :, 2] = 0.0
        W0[7] *= 1e307
        fr = FrameSpec(8, chain, W0)
        a = _run(sysm, x0, 300, fr, 5, "fp64", V_ONE)
        b = _run(sysm, x0, 300, fr, 5, "fp64", V_COOP)
        _same(a, b)
        assert a.code[3] == 1 and a.code[5] == 3 and a.code[7] != 0
