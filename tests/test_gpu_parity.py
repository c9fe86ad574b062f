"""Parity of the B200 FP64 kernels with the CPU oracle, bit for bit.

The plain (FP64) kernels evaluate the reference's arithmetic operation for operation with the same portable
sin / cos / log as the oracle's MATH_PORTABLE mode, so every record -- final point, frames, the reducer states in
the Julia layout, status codes and failing steps -- must agree bitwise on the same inputs, chaotic orbits
included. Each case runs the same seeded inputs through `chaos_b200.propagate_frames` (the C ABI on the GPU) and
`oracle.oracle_frames` (serial C++ on the CPU).
"""
from __future__ import annotations

import numpy as np
import pytest

from chaos_b200 import (CGS, FLI, GALI, MEGNO, MGS, RGS, SALI, AugmentedQR, Benettin, FroeschleMap, GivensQR,
                        HouseholderQR, LinearSymplecticMap, QRSpectrum, StandardMap, StandardMapChain,
                        WrappedStandardMap, propagate_frames, torus_state)
from chaos_b200.propagate import FrameSpec
from helpers import haar_frames, identity_frames, same_bits, states_equal, uniform_starts

pytestmark = pytest.mark.gpu

QRS = [CGS(), MGS(), RGS(), HouseholderQR(), AugmentedQR(), GivensQR()]


def _compare(sys, x0, N, frames, tau, oracle, launch_steps=None, seed=7):
    dev = propagate_frames(sys, x0, N, frames, tau=tau, seed=seed, finals=False, throw=False,
                           launch_steps=launch_steps)
    ref = oracle.oracle_frames(sys, x0, N, frames, tau=tau, seed=seed, math="portable")
    for f in range(len(frames)):
        assert same_bits(dev[f].x, ref[f]["x"]), f"x differs (frame {f})"
        assert np.array_equal(dev[f].code, ref[f]["code"]), f"code differs (frame {f})"
        assert np.array_equal(dev[f].hstep, ref[f]["hstep"]), f"hstep differs (frame {f})"
        assert same_bits(dev[f].W, ref[f]["W"]), f"W differs (frame {f})"
        assert states_equal(dev[f].states, ref[f]["states"]), f"states differ (frame {f})"
    return dev, ref


def _chains_k2():
    return [(QRSpectrum(a),) for a in QRS] + [(SALI(),), (GALI(),), (MEGNO(),), (FLI(),),
                                              (MEGNO(replace=False), FLI(replace=False), QRSpectrum(GivensQR())),
                                              (MEGNO(replace=False), SALI()), (FLI(replace=False), SALI()),
                                              (MEGNO(replace=False), FLI(replace=False), SALI()), ()]


@pytest.mark.parametrize("chain", [(Benettin(),)] + [(QRSpectrum(a),) for a in QRS], ids=repr)
@pytest.mark.parametrize("wrapped", [False, True])
def test_standard_k1(oracle, chain, wrapped):
    n = 257
    z = uniform_starts(n, 2, 11)
    sys = WrappedStandardMap(6.0) if wrapped else StandardMap(6.0)
    x0 = np.array([torus_state(v) for v in z]) if wrapped else z
    W0 = haar_frames(n, 2, 1, 12)
    _compare(sys, x0, 3000, [FrameSpec(1, chain, W0)], 1, oracle)


@pytest.mark.parametrize("chain", _chains_k2(), ids=repr)
@pytest.mark.parametrize("wrapped", [False, True])
def test_standard_k2(oracle, chain, wrapped):
    n = 300
    z = uniform_starts(n, 2, 21)
    sys = WrappedStandardMap(6.0) if wrapped else StandardMap(6.0)
    x0 = np.array([torus_state(v) for v in z]) if wrapped else z
    W0 = identity_frames(n, 2, 2)
    _compare(sys, x0, 4000, [FrameSpec(2, chain, W0)], 1, oracle)


@pytest.mark.parametrize("tau", [1, 5, 10])
def test_standard_tau_and_relaunch(oracle, tau):
    n = 200
    x0 = uniform_starts(n, 2, 31)
    fr = [FrameSpec(2, (QRSpectrum(MGS()),), haar_frames(n, 2, 2, 32))]
    one, _ = _compare(StandardMap(1.5), x0, 2000, fr, tau, oracle)
    # step-chunked relaunch carrying the state (propagate.jl:101-109) gives the same bits
    many, _ = _compare(StandardMap(1.5), x0, 2000, fr, tau, oracle, launch_steps=10 * tau)
    assert same_bits(one[0].W, many[0].W) and states_equal(one[0].states, many[0].states)


@pytest.mark.parametrize("k,chain", [(1, (Benettin(),)), (1, (QRSpectrum(MGS()),))]
                         + [(2, c) for c in _chains_k2()]
                         + [(k, (QRSpectrum(a),)) for k in (3, 4) for a in QRS]
                         + [(k, (GALI(),)) for k in (3, 4)] + [(4, (GALI(), SALI()))], ids=repr)
def test_froeschle(oracle, k, chain):
    n = 256
    x0 = uniform_starts(n, 4, 41)
    W0 = haar_frames(n, 4, k, 42)
    _compare(FroeschleMap(1.5, 1.5, 0.05), x0, 2000, [FrameSpec(k, chain, W0)], 10, oracle)


def test_froeschle_fused_frames(oracle):
    """QRSpectrum(Householder) and GALI_4 + SALI carried along one orbit (the coupled-maps ensemble)."""
    n = 512
    x0 = uniform_starts(n, 4, 51)
    W0 = identity_frames(n, 4, 4)
    frames = [FrameSpec(4, (QRSpectrum(HouseholderQR()),), W0), FrameSpec(4, (GALI(), SALI()), W0)]
    dev, _ = _compare(FroeschleMap(1.5, 1.5, 0.05), x0, 5000, frames, 10, oracle)
    # each frame equals its own single-frame run (a separate reference call on the same orbit and W0)
    for f in range(2):
        single = propagate_frames(FroeschleMap(1.5, 1.5, 0.05), x0, 5000, [frames[f]], tau=10, finals=False,
                                  throw=False)[0]
        assert same_bits(single.W, dev[f].W) and states_equal(single.states, dev[f].states)


@pytest.mark.parametrize("N_sites", range(2, 9))
@pytest.mark.parametrize("ring", [False, True])
def test_chain(oracle, N_sites, ring):
    if ring and N_sites < 3:
        pytest.skip("a ring needs N >= 3")
    d = 2 * N_sites
    n = 128
    sys = StandardMapChain(N_sites, 1.2, 0.05, boundary="ring" if ring else "open")
    x0 = uniform_starts(n, d, 60 + N_sites)
    k = min(d, 8)
    for chain in ((QRSpectrum(MGS()),), (QRSpectrum(HouseholderQR()),), (GALI(),)):
        _compare(sys, x0, 500, [FrameSpec(k, chain, haar_frames(n, d, k, 70))], 5, oracle)
    for chain in ((QRSpectrum(MGS()),), (SALI(),), (MEGNO(),)):
        _compare(sys, x0, 500, [FrameSpec(2, chain, haar_frames(n, d, 2, 71))], 5, oracle)


@pytest.mark.parametrize("k,chain", [(1, (Benettin(),)), (2, (QRSpectrum(MGS()),)), (2, (MEGNO(),)), (2, (SALI(),))],
                         ids=repr)
def test_linear(oracle, k, chain):
    A = np.array([[2.0, 1.0], [1.0, 1.0]])
    n = 64
    x0 = uniform_starts(n, 2, 80, -1, 1)
    _compare(LinearSymplecticMap(A), x0, 300, [FrameSpec(k, chain, haar_frames(n, 2, k, 81))], 1, oracle)


def test_seeded_frames(oracle):
    """W0 = nothing: the seeded Haar frames are drawn on the device, bit-identical to the oracle's stream."""
    n = 300
    x0 = uniform_starts(n, 4, 90)
    _compare(FroeschleMap(1.5, 1.5, 0.05), x0, 200, [FrameSpec(4, (QRSpectrum(MGS()),), None)], 10, oracle,
             seed=123)


def test_failures_match(oracle):
    """Orbits that fail -- non-finite start (STATUS_STATE), overflowing frame (STATUS_W), a zero column
    (QR pivot breakdown) -- report the same code, step and reducer record."""
    n = 64
    x0 = uniform_starts(n, 2, 100)
    x0[3, 0] = np.nan
    W0 = haar_frames(n, 2, 2, 101)
    W0[5, :, 1] = 0.0                       # zero second column: MGS pivot failure at the first handoff
    W0[7] *= 1e307                          # overflows within the first handoff interval (K = 6)
    for chain in ((QRSpectrum(MGS()),), (QRSpectrum(HouseholderQR()),), (SALI(),), (MEGNO(),), (FLI(),), (GALI(),)):
        dev, ref = _compare(StandardMap(6.0), x0, 50, [FrameSpec(2, chain, W0)], 5, oracle)
        assert dev[0].code[3] == 1 and dev[0].code[7] in (2, 3)


@pytest.mark.parametrize("k,chain", [(2, (MEGNO(replace=False), FLI(replace=False), QRSpectrum(GivensQR()))),
                                     (2, (QRSpectrum(MGS()),)), (2, (SALI(),)), (4, (QRSpectrum(HouseholderQR()),)),
                                     (4, (GALI(),)), (1, (Benettin(),))], ids=repr)
@pytest.mark.parametrize("tol", [1e-14, None])
def test_henon_heiles_gauss3(oracle, k, chain, tol):
    """IntegratorMap(Gauss(Float64, 3; tol), HenonHeilesFlow(), 0.01): the fixed-point solve, the 12 x 12 tangent
    solve and the reducers, bit for bit against the oracle, on E = 1/8 energy-shell starts."""
    from chaos_b200 import Gauss, HenonHeilesFlow, IntegratorMap, random_energy_starts
    n = 96
    x0 = random_energy_starts(1 / 8, n, seed=5)
    sysm = IntegratorMap(Gauss(3, tol=tol), HenonHeilesFlow(), 0.01)
    _compare(sysm, x0, 600, [FrameSpec(k, chain, haar_frames(n, 4, k, 6))], 10, oracle)


@pytest.mark.parametrize("k,chain", [(2, (MEGNO(replace=False), FLI(replace=False), QRSpectrum(GivensQR()))),
                                     (2, (QRSpectrum(MGS()),)), (2, (SALI(),)), (4, (QRSpectrum(HouseholderQR()),)),
                                     (4, (GALI(),)), (1, (Benettin(),))], ids=repr)
@pytest.mark.parametrize("method", ["KahanLi8", "KahanLi6", "LeapfrogKDK", "SABA4", "SBAB3", "Ruth3", "CalvoSanzSerna4",
                                    "SymplecticEulerKD", "SofroniouSpaletta10", "Suzuki8", "ABAH864", "SABAC2",
                                    "SBABC3"])
def test_henon_heiles_splitting(oracle, k, chain, method):
    """IntegratorMap(SplittingMethod, HenonHeilesFlow(), 0.05): merged-kick forward, the stage-Jacobian tangent and the
    reducers, bit for bit against the oracle on E = 1/8 energy-shell starts."""
    import chaos_b200 as cb
    from chaos_b200 import HenonHeilesFlow, IntegratorMap, random_energy_starts
    m = {"KahanLi8": lambda: cb.KahanLi(8), "KahanLi6": lambda: cb.KahanLi(6), "LeapfrogKDK": lambda: cb.Leapfrog("KDK"),
         "SABA4": lambda: cb.SABA(4), "SBAB3": lambda: cb.SBAB(3), "Ruth3": cb.Ruth3, "CalvoSanzSerna4": cb.CalvoSanzSerna4,
         "SymplecticEulerKD": lambda: cb.SymplecticEuler("KD"), "SofroniouSpaletta10": cb.SofroniouSpaletta10,
         "Suzuki8": lambda: cb.suzuki_jump(cb.Leapfrog(), 8), "ABAH864": cb.ABAH864, "SABAC2": lambda: cb.SABAC(2),
         "SBABC3": lambda: cb.SBABC(3)}[method]()
    n = 160
    x0 = random_energy_starts(1 / 8, n, seed=12)
    sysm = IntegratorMap(m, HenonHeilesFlow(), 0.05)
    _compare(sysm, x0, 800, [FrameSpec(k, chain, haar_frames(n, 4, k, 13))], 10, oracle)


def test_propagate_orbit(oracle):
    """propagate_orbit (src/Tangent/orbit.jl:77-99): one orbit through the kernel, the oracle's bits, and the
    errors of a failing orbit naming the orbit id the caller gives."""
    from chaos_b200 import NumericalHealthError, propagate_orbit
    x0 = np.array([0.3, 1.1, 2.0, 0.7])
    W0 = haar_frames(1, 4, 4, 3)[0]
    sysm = FroeschleMap(1.5, 1.5, 0.05)
    x, W, st = propagate_orbit(sysm, x0, W0, 1000, 10, (QRSpectrum(HouseholderQR()),))
    ref = oracle.oracle_frames(sysm, x0[None], 1000, [FrameSpec(4, (QRSpectrum(HouseholderQR()),), W0[None])], tau=10,
                               math="portable")[0]
    assert same_bits(x, ref["x"][0]) and same_bits(W, ref["W"][0]) and states_equal(st[None], ref["states"])
    with pytest.raises(NumericalHealthError) as e:
        propagate_orbit(sysm, np.array([np.nan, 0.0, 0.0, 0.0]), W0, 100, 10, (QRSpectrum(MGS()),), orbit=7)
    assert e.value.orbit == 7 and e.value.what == "state" and e.value.step == 10
    with pytest.raises(NumericalHealthError) as e:
        propagate_orbit(StandardMap(6.0), np.array([0.1, 0.2]), np.zeros((2, 2)), 50, 5, (QRSpectrum(MGS()),), orbit=3)
    assert e.value.orbit == 3


@pytest.mark.parametrize("method", ["KahanLi8", "SABAC2"])
def test_henon_heiles_splitting_mixed(method):
    """The mixed splitting kernel (Float64 orbit and stage states, Float32 tangent from the stage Jacobians'
    blocks): the orbit bit for bit the plain kernel's, lambda_1 within 1e-3 of the plain kernel's."""
    import chaos_b200 as cb
    from chaos_b200 import HenonHeilesFlow, IntegratorMap, random_energy_starts
    m = {"KahanLi8": lambda: cb.KahanLi(8), "SABAC2": lambda: cb.SABAC(2)}[method]()
    n, N = 512, 20000
    x0 = random_energy_starts(1 / 8, n, seed=21)
    sysm = IntegratorMap(m, HenonHeilesFlow(), 0.05)
    for k, chain in ((2, (MEGNO(replace=False), FLI(replace=False), QRSpectrum(GivensQR()))),
                     (4, (QRSpectrum(HouseholderQR()),))):
        fr = [FrameSpec(k, chain, identity_frames(n, 4, k))]
        a = propagate_frames(sysm, x0, N, fr, tau=10, finals=False, throw=False)[0]
        b = propagate_frames(sysm, x0, N, fr, tau=10, precision="mixed", finals=False, throw=False)[0]
        assert same_bits(a.x, b.x)
        key = "r2" if k == 2 else "r0"
        la = (a.states[key]["sums"][:, 0, 0] + a.states[key]["sums"][:, 0, 1]) / N
        lb = (b.states[key]["sums"][:, 0, 0] + b.states[key]["sums"][:, 0, 1]) / N
        ok = (a.code == 0) & (b.code == 0)
        assert ok.mean() > 0.99 and np.max(np.abs(la[ok] - lb[ok])) <= 1e-3


@pytest.mark.parametrize("dt", [0.01, 0.05])
def test_henon_heiles_gauss3_mixed(dt):
    """The mixed Gauss kernel (the Float64 step, the tangent's linear system in Float32 by its fixed-point form):
    the orbit bit for bit the plain kernel's, lambda_1 and the MEGNO average within 1e-3 of the plain kernel's."""
    from chaos_b200 import Gauss, HenonHeilesFlow, IntegratorMap, random_energy_starts
    n, N = 512, 20000
    x0 = random_energy_starts(1 / 8, n, seed=23)
    sysm = IntegratorMap(Gauss(3, tol=1e-14), HenonHeilesFlow(), dt)
    chain = (MEGNO(replace=False), FLI(replace=False), QRSpectrum(GivensQR()))
    fr = [FrameSpec(2, chain, identity_frames(n, 4, 2))]
    a = propagate_frames(sysm, x0, N, fr, tau=10, finals=False, throw=False)[0]
    b = propagate_frames(sysm, x0, N, fr, tau=10, precision="mixed", finals=False, throw=False)[0]
    assert same_bits(a.x, b.x)
    la = (a.states["r2"]["sums"][:, 0, 0] + a.states["r2"]["sums"][:, 0, 1]) / N
    lb = (b.states["r2"]["sums"][:, 0, 0] + b.states["r2"]["sums"][:, 0, 1]) / N
    ok = (a.code == 0) & (b.code == 0)
    assert ok.mean() > 0.99 and np.max(np.abs(la[ok] - lb[ok])) <= 1e-3
