"""The statically sized oracle (oracle/static_leg.cpp, the timed CPU baseline): its records are bit for bit the
runtime-sized oracle's on the configurations it covers, carried relaunches and failures included."""
import numpy as np
import pytest

from chaos_b200 import (FLI, GALI, MEGNO, MGS, SALI, Benettin, FroeschleMap, GivensQR, HouseholderQR, QRSpectrum,
                        StandardMap, WrappedFroeschleMap, WrappedStandardMap)
from chaos_b200.propagate import FrameSpec
from helpers import haar_frames, identity_frames, same_bits, states_equal, uniform_starts


def _same(a, b):
    for fa, fb in zip(a, b):
        assert same_bits(fa["x"], fb["x"]) and same_bits(fa["W"], fb["W"])
        assert states_equal(fa["states"], fb["states"])
        assert np.array_equal(fa["code"], fb["code"]) and np.array_equal(fa["hstep"], fb["hstep"])


CASES = [
    ("c1", lambda: WrappedStandardMap(6.0), 2, lambda n: [FrameSpec(2, (QRSpectrum(MGS()),), identity_frames(n, 2, 2))], 1),
    ("std-k1", lambda: StandardMap(1.2), 2, lambda n: [FrameSpec(1, (Benettin(),), identity_frames(n, 2, 1))], 5),
    ("c2", lambda: FroeschleMap(1.5, 1.5, 0.05), 4,
     lambda n: [FrameSpec(4, (QRSpectrum(HouseholderQR()),), identity_frames(n, 4, 4)),
                FrameSpec(4, (GALI(), SALI()), identity_frames(n, 4, 4))], 10),
    ("fro-k2", lambda: FroeschleMap(1.5, 1.5, 0.05), 4,
     lambda n: [FrameSpec(2, (MEGNO(replace=False), FLI(replace=False), QRSpectrum(GivensQR())), haar_frames(n, 4, 2, 5))], 4),
    ("wfro", lambda: WrappedFroeschleMap(1.5, 1.5, 0.05), 4,
     lambda n: [FrameSpec(4, (QRSpectrum(HouseholderQR()),), identity_frames(n, 4, 4))], 10),
]


@pytest.mark.parametrize("name,mk,d,frames,tau", CASES, ids=[c[0] for c in CASES])
def test_static_equals_runtime(oracle, name, mk, d, frames, tau):
    n, N = 48, 600
    sysm = mk()
    z = uniform_starts(n, d, seed=3)
    x0 = np.array([sysm.torus_state(zi) for zi in z]) if sysm.s > d else z
    x0[5] = np.nan   # a failing orbit
    fr = frames(n)
    ref = oracle.oracle_frames(sysm, x0, N, fr, tau=tau, math="portable", threads=2)
    got = oracle.oracle_frames(sysm, x0, N, fr, tau=tau, math="portable", threads=3, engine="static")
    _same(got, ref)
    relaunch = oracle.oracle_frames(sysm, x0, N, fr, tau=tau, math="portable", threads=2, engine="static",
                                    launch_steps=tau * 7)
    _same(relaunch, ref)


def test_static_rejects_uncovered(oracle):
    sysm = FroeschleMap(1.5, 1.5, 0.05)
    x0 = uniform_starts(4, 4, seed=1)
    fr = [FrameSpec(4, (QRSpectrum(HouseholderQR()),), identity_frames(4, 4, 4)),
          FrameSpec(2, (SALI(),), identity_frames(4, 4, 2))]
    with pytest.raises(ValueError):
        oracle.oracle_frames(sysm, x0, 20, fr, tau=10, engine="static")
