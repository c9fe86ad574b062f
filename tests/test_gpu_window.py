"""The indicator recorder's window kinds on the B200 against the oracle, bit for bit: the rows, the failing grid
index, the carried point, the monitor's and the reader's states (so every final), status and failing step, for the
weighted phase advance (planar and lifted-angle observables) and the weighted Birkhoff averages (cos, sin, lifted
and coordinate observables), one to three horizons, Birkhoff orders 1 to 4, three systems, tau 1 and 3, in one
launch and in windows, with failures."""
from __future__ import annotations

import numpy as np
import pytest

from chaos_b200 import LinearSymplecticMap, StandardMap, WrappedStandardMap, torus_state
from chaos_b200.window import (CosObservable, IndCoordinate, LiftedAngleObservable, LiftedObservable,
                               PlanarObservable, SinObservable, WeightedBirkhoff, WeightedPhaseAdvance,
                               record_indicator_window)
from helpers import same_bits

pytestmark = pytest.mark.gpu


def _system(name, n=200):
    z = np.random.default_rng(51).uniform(0, 2 * np.pi, (n, 2))
    if name == "standard":
        return StandardMap(1.1), z
    if name == "wrapped":
        return WrappedStandardMap(3.5), np.array([torus_state(v) for v in z])
    return LinearSymplecticMap([[0.6, -0.8], [0.8, 0.6]]), z


def _readers(name):
    wrapped = name == "wrapped"
    lifted_angle = LiftedAngleObservable(1, 3) if wrapped else LiftedAngleObservable(1)
    coord = LiftedObservable(2, 4) if wrapped else IndCoordinate(2)
    return {
        "pa-planar": WeightedPhaseAdvance(window=(40, 16), observable=PlanarObservable(1, 2)),
        "pa-lifted-p3": WeightedPhaseAdvance(window=32, observable=lifted_angle, birkhoff_order=3),
        "wb-trig": WeightedBirkhoff(window=(24, 48, 16), observables=(CosObservable(1), SinObservable(1, 2),
                                                                      CosObservable(2, 3))),
        "wb-coord-p2": WeightedBirkhoff(window=40, observables=(coord, SinObservable(2)), birkhoff_order=2),
        "wb-p4": WeightedBirkhoff(window=(16, 20), observables=(CosObservable(1),), birkhoff_order=4),
    }


def _same(dev, ref):
    assert same_bits(dev.R, ref["R"]), "R"
    assert same_bits(dev.x, ref["x"]), "x"
    w1 = np.ascontiguousarray(dev.states).view(np.uint64).copy()
    w2 = np.ascontiguousarray(ref["states"]).view(np.uint64).copy()
    for w in (w1, w2):
        w[np.isnan(w.view(np.float64))] = 0x7FF8000000000000
    assert np.array_equal(w1, w2), "states"
    for key in ("fail", "code", "hstep"):
        assert np.array_equal(getattr(dev, key), ref[key]), key


@pytest.mark.parametrize("reader", ["pa-planar", "pa-lifted-p3", "wb-trig", "wb-coord-p2", "wb-p4"])
@pytest.mark.parametrize("name", ["standard", "wrapped", "linear"])
@pytest.mark.parametrize("tau", [1, 3])
def test_window_matches_oracle(oracle, reader, name, tau):
    sys, x0 = _system(name)
    red = _readers(name)[reader]
    N = tau * red.handoffs()
    grid = sorted({g for g in (tau, 4 * tau, 16 * tau, N) if g <= N})
    dev = record_indicator_window(sys, x0, N, tau, red, grid, ns=sys.s)
    ref = oracle.oracle_indicator_window(sys, x0, N, tau, red, grid, ns=sys.s)
    _same(dev, ref)


@pytest.mark.parametrize("L", [5, 31])
def test_window_launch_windows(oracle, L):
    sys, x0 = _system("wrapped")
    red = _readers("wrapped")["wb-trig"]
    N = red.handoffs()
    grid = [1, 5, 50, N]
    dev = record_indicator_window(sys, x0, N, 1, red, grid, ns=4, launch_steps=L)
    ref = oracle.oracle_indicator_window(sys, x0, N, 1, red, grid, ns=4)
    _same(dev, ref)


def test_window_failures(oracle):
    x0 = np.array([[0.3, 0.2], [0.5, 1e308], [1.0, 0.5], [np.nan, 0.0]])
    red = WeightedBirkhoff(window=16, observables=(IndCoordinate(1), LiftedObservable(1, 2)))
    dev = record_indicator_window(StandardMap(0.0), x0, 32, 1, red, [4, 16, 32])
    ref = oracle.oracle_indicator_window(StandardMap(0.0), x0, 32, 1, red, [4, 16, 32])
    _same(dev, ref)
    assert dev.fail.tolist() == [0, 1, 0, 1] and dev.code.tolist() == [0, 3, 0, 1]
    red = WeightedPhaseAdvance(window=16, observable=PlanarObservable(1, 2))
    z = np.array([[0.0, 0.0], [1.0, 2.0]])
    dev = record_indicator_window(LinearSymplecticMap([[2.0, 1.0], [1.0, 1.0]]), z, 33, 1, red, [33])
    ref = oracle.oracle_indicator_window(LinearSymplecticMap([[2.0, 1.0], [1.0, 1.0]]), z, 33, 1, red, [33])
    _same(dev, ref)
    assert np.isnan(dev.finals[0]["nu1"][0]) and dev.code[0] == 0
