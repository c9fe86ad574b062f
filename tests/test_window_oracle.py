"""The indicator recorder's window kinds on the oracle (CPU): the reference's weighted-Birkhoff known answers
(test/weighted-birkhoff/wb_ac01_03.jl: AC1a a constant observable gives both averages equal, Delta = 0 bitwise, the
floor flag; AC3 the K = 0 standard map gives cos q, sin q averages within 4 eps, |Delta| <= 8 eps, the lifted p equal
to p_0), the phase advance of exact rotations (the lifted angle of the K = 0 map and the planar angle of a rotation
matrix, nu = angle / 2 pi), the planar origin (an undefined frequency without a failure, test/naff-fma/nf_d81.jl:90),
frozen horizons, failures, launch windows, and the monitor rows against the study recorder's."""
from __future__ import annotations

import math

import numpy as np
import pytest

from chaos_b200 import MGS, LinearSymplecticMap, QRSpectrum, StandardMap, WrappedStandardMap, torus_state
from chaos_b200.window import (CosObservable, IndCoordinate, LiftedAngleObservable, LiftedObservable,
                               PlanarObservable, SinObservable, WeightedBirkhoff, WeightedPhaseAdvance,
                               record_indicator_window)

EPS = 2.0 ** -52


@pytest.mark.parametrize("N", [1000, 4000])
def test_zero_shear_birkhoff(oracle, N):
    sys = WrappedStandardMap(0.0)
    rng = np.random.default_rng(3)
    for p0 in (1.0, 2.0, 3.3, 5.0):
        q0s = 2 * np.pi * rng.random(4)
        x0 = np.array([torus_state([q, p0]) for q in q0s])
        red = WeightedBirkhoff(window=N, observables=(CosObservable(1), SinObservable(1), LiftedObservable(2, 4)))
        rec = oracle.oracle_indicator_window(sys, x0, 2 * N, 1, red, [N, 2 * N])
        for f in rec["finals"]:
            assert f["complete"]
            for k in range(2):
                assert abs(f["avg1"][k, 0]) <= 4 * EPS and abs(f["avg2"][k, 0]) <= 4 * EPS
                assert abs(f["delta"][k, 0]) <= 8 * EPS
            assert abs(f["avg1"][2, 0] - p0) <= 2 * EPS * p0 and abs(f["avg2"][2, 0] - p0) <= 2 * EPS * p0
    q0s = 2 * np.pi * rng.random(4)        # p0 = pi: cos 2q is the constant cos 2 q0
    x0 = np.array([torus_state([q, math.pi]) for q in q0s])
    rec = oracle.oracle_indicator_window(sys, x0, 2 * N, 1, WeightedBirkhoff(window=N, observables=(CosObservable(1, 2),)),
                                         [2 * N])
    for q0, f in zip(q0s, rec["finals"]):
        c = math.cos(2 * torus_state([q0, math.pi])[0])
        assert abs(f["avg1"][0, 0] - c) <= 16 * EPS and abs(f["delta"][0, 0]) <= 8 * EPS


@pytest.mark.parametrize("c", [0.3, 1e3, 1e-3, math.pi])
def test_constant_observable(oracle, c):
    sys = StandardMap(0.0)
    N = 1000
    red = WeightedBirkhoff(window=(N, 2 * N), observables=(IndCoordinate(2),))
    rec = oracle.oracle_indicator_window(sys, np.array([[1.0, c]]), 4 * N, 1, red, [4 * N])
    f = rec["finals"][0]
    for h in range(2):
        assert abs(f["avg1"][0, h] - c) <= 2 * EPS * c and abs(f["avg2"][0, h] - c) <= 2 * EPS * c
        assert f["delta"][0, h] == 0 and f["below_floor"][0, h] and not f["zero"][0, h] and f["S"][0, h] == c
        ref = -math.log10(32 * EPS * c)
        assert abs(f["absdig"][0, h] - ref) <= 2 * EPS * abs(ref) + 1e-15


def test_phase_advance_of_rotations(oracle):
    red = WeightedPhaseAdvance(window=(500, 250), observable=LiftedAngleObservable(1, 3))
    p0s = [0.25, 1.234, 2.9]
    x0 = np.array([torus_state([0.3, p]) for p in p0s])
    rec = oracle.oracle_indicator_window(WrappedStandardMap(0.0), x0, 1001, 1, red, [1001])
    for p, f in zip(p0s, rec["finals"]):
        assert f["complete"] and f["near_pi"] == 0
        for h in range(2):
            assert abs(f["nu1"][h] - p / (2 * math.pi)) <= 8 * EPS and abs(f["nu2"][h] - p / (2 * math.pi)) <= 8 * EPS
            assert f["below_floor"][h]
    for th in (0.7, 2.0, -1.1, 3.0):
        A = [[math.cos(th), -math.sin(th)], [math.sin(th), math.cos(th)]]
        red = WeightedPhaseAdvance(window=300, observable=PlanarObservable(1, 2))
        rec = oracle.oracle_indicator_window(LinearSymplecticMap(A), np.array([[1.0, 0.5], [-0.2, 3.0]]), 601, 1, red,
                                             [601])
        for f in rec["finals"]:
            assert abs(f["nu1"][0] - th / (2 * math.pi)) <= 64 * EPS and abs(f["nu2"][0] - th / (2 * math.pi)) <= 64 * EPS
            assert f["near_pi"] == (600 if abs(th) > 0.9 * math.pi else 0)


def test_planar_origin_is_undefined_not_failed(oracle):
    red = WeightedPhaseAdvance(window=16, observable=PlanarObservable(1, 2))
    rec = oracle.oracle_indicator_window(LinearSymplecticMap([[2.0, 1.0], [1.0, 1.0]]), np.zeros((1, 2)), 33, 1, red,
                                         [33])
    f = rec["finals"][0]
    assert rec["code"][0] == 0 and rec["fail"][0] == 0
    assert math.isnan(f["nu1"][0]) and math.isnan(f["nu2"][0]) and math.isnan(f["D"][0]) and not f["below_floor"][0]


def test_frozen_horizons_change_nothing(oracle):
    sys = StandardMap(0.9)
    x0 = np.random.default_rng(5).uniform(0, 2 * np.pi, (8, 2))
    red = WeightedBirkhoff(window=(20, 40), observables=(CosObservable(1), SinObservable(2, 3)), birkhoff_order=2)
    a = oracle.oracle_indicator_window(sys, x0, 80, 1, red, [80])
    b = oracle.oracle_indicator_window(sys, x0, 120, 1, red, [80])
    for fa, fb in zip(a["finals"], b["finals"]):
        for key in ("avg1", "avg2", "S", "B"):
            assert np.array_equal(fa[key], fb[key], equal_nan=True)
        assert fb["handoffs"] == 120 and fb["n"] == 120


@pytest.mark.parametrize("L", [3, 30, 99])
@pytest.mark.parametrize("kind", ["pa", "wb"])
def test_launch_windows_change_no_bit(oracle, L, kind):
    sys = WrappedStandardMap(1.7)
    x0 = np.array([torus_state(v) for v in np.random.default_rng(6).uniform(0, 2 * np.pi, (12, 2))])
    red = WeightedPhaseAdvance(window=(16, 32), observable=PlanarObservable(1, 2), birkhoff_order=3) if kind == "pa" \
        else WeightedBirkhoff(window=(16, 32), observables=(CosObservable(1), LiftedObservable(2, 4)), birkhoff_order=4)
    N = 3 * red.handoffs()
    a = oracle.oracle_indicator_window(sys, x0, N, 3, red, [3, 60, N], ns=4)
    b = oracle.oracle_indicator_window(sys, x0, N, 3, red, [3, 60, N], ns=4, launch_steps=L)
    for key in ("R", "fail", "x", "states", "code", "hstep"):
        assert np.asarray(a[key]).tobytes() == np.asarray(b[key]).tobytes(), key


def test_failures(oracle):
    sys = StandardMap(1.0)
    x0 = np.array([[0.3, 0.2], [0.5, 1e308], [1.0, 0.5]])
    red = WeightedBirkhoff(window=16, observables=(IndCoordinate(2),))
    rec = oracle.oracle_indicator_window(sys, x0, 32, 1, red, [4, 16, 32])
    assert rec["fail"].tolist() == [0, 1, 0] and rec["code"].tolist() == [0, 1, 0] and rec["hstep"][1] == 2
    # a non-finite observable value: the lifted observable on a winding count near the float range (x + 2 pi m)
    z = np.array([[0.5, 1e308]])
    red = WeightedBirkhoff(window=16, observables=(IndCoordinate(1), LiftedObservable(1, 2)))
    rec = oracle.oracle_indicator_window(StandardMap(0.0), z, 32, 1, red, [16, 32])
    assert rec["code"][0] == 3 and rec["fail"][0] == 1
    tail = 16 + 40 * 2                      # H (16 + 40 K): the code field follows n and handoffs
    assert int(np.frombuffer(rec["states"][0, 24 + tail + 12: 24 + tail + 14].tobytes(), "<i2")[0]) == 2


def test_monitor_rows_are_the_recorders(oracle):
    sys = WrappedStandardMap(2.5)
    x0 = np.array([torus_state(v) for v in np.random.default_rng(8).uniform(0, 2 * np.pi, (10, 2))])
    red = WeightedBirkhoff(window=25, observables=(SinObservable(1),))
    grid = [5, 25, 50]
    w = oracle.oracle_indicator_window(sys, x0, 50, 1, red, grid, ns=4)
    r = oracle.oracle_record(sys, x0, 50, 1, QRSpectrum(MGS()), grid)
    assert np.array_equal(w["R"][:, :, 0], r["R"][:, :, 2]) and np.array_equal(w["R"][:, :, 1], r["R"][:, :, 3])
    assert np.array_equal(w["R"][:, :, 2], r["R"][:, :, 8]) and np.array_equal(w["R"][:, :, 3:], r["R"][:, :, 9:])


def test_host_checks():
    with pytest.raises(ValueError):
        WeightedBirkhoff(window=15, observables=(CosObservable(1),))
    with pytest.raises(ValueError):
        WeightedPhaseAdvance(window=16, observable=PlanarObservable(1, 2), birkhoff_order=5)
    with pytest.raises(ValueError):
        WeightedBirkhoff(window=16, observables=())
    red = WeightedPhaseAdvance(window=16, observable=PlanarObservable(1, 2))
    with pytest.raises(ValueError, match="handoffs"):
        record_indicator_window(StandardMap(1.0), np.zeros((2, 2)), 32, 1, red, [32])
