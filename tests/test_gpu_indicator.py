"""The indicator recorder (tangent kind) on the B200 against the oracle, bit for bit: every row of R, the failing
grid index, the carried point, frame, member and monitor states, status and failing step, for every compiled member
chain on the lifted and wrapped standard maps and a linear map, tau 1 and 4, in one launch and in windows."""
from __future__ import annotations

import numpy as np
import pytest

from chaos_b200 import LinearSymplecticMap, StandardMap, WrappedStandardMap, record_indicators, torus_state
from helpers import same_bits

pytestmark = pytest.mark.gpu

CHAINS = [["SALI"], ["FLI", "SALI"], ["MEGNO", "SALI"], ["FLI", "MEGNO", "SALI"], ["FLI"], ["MEGNO"], ["FLI", "MEGNO"],
          ["MEGNO", "FLI", "SALI"], ["MEGNO", "FLI"], ["SALI", "MEGNO"], ["SALI", "FLI"]]


def _system(name):
    z = np.random.default_rng(37).uniform(0, 2 * np.pi, (160, 2))
    if name == "standard":
        return StandardMap(2.5), z
    if name == "wrapped":
        return WrappedStandardMap(6.0), np.array([torus_state(v) for v in z])
    return LinearSymplecticMap([[2.0, 1.0], [1.0, 1.0]]), z * 1e-6


def _words(a):
    w = np.ascontiguousarray(a).view(np.uint64).copy()
    w[np.isnan(w.view(np.float64))] = 0x7FF8000000000000
    return w


def _same(dev, ref):
    assert same_bits(dev.R, ref["R"]), "R"
    assert same_bits(dev.x, ref["x"]) and same_bits(dev.W, ref["W"]), "x / W"
    assert np.array_equal(_words(dev.states), _words(ref["states"])), "states"
    for key in ("fail", "code", "hstep"):
        assert np.array_equal(getattr(dev, key), ref[key]), key


@pytest.mark.parametrize("members", CHAINS, ids=",".join)
@pytest.mark.parametrize("name", ["standard", "wrapped", "linear"])
@pytest.mark.parametrize("tau", [1, 4])
def test_indicator_matches_oracle(oracle, members, name, tau):
    sys, x0 = _system(name)
    N = 200 if name != "linear" else 40
    grid = sorted({g for g in (tau, 2 * tau, 10 * tau, 25 * tau, N) if g <= N})
    ns = sys.s
    dev = record_indicators(sys, x0, N, tau, members, grid, ns=ns)
    ref = oracle.oracle_indicators(sys, x0, N, tau, members, grid, ns=ns)
    _same(dev, ref)


@pytest.mark.parametrize("L", [8, 48])
def test_indicator_windows(oracle, L):
    sys, x0 = _system("wrapped")
    grid = [8, 16, 40, 96, 200]
    dev = record_indicators(sys, x0, 200, 4, ["FLI", "MEGNO", "SALI"], grid, ns=2, launch_steps=L)
    ref = oracle.oracle_indicators(sys, x0, 200, 4, ["FLI", "MEGNO", "SALI"], grid, ns=2)
    _same(dev, ref)


def test_indicator_failure(oracle):
    sys = StandardMap(1.0)
    x0 = np.array([[0.3, 0.2], [0.5, 1e308], [1.0, 0.5], [np.nan, 0.1]])
    grid = [2, 4, 8]
    dev = record_indicators(sys, x0, 8, 2, ["MEGNO", "SALI"], grid)
    ref = oracle.oracle_indicators(sys, x0, 8, 2, ["MEGNO", "SALI"], grid)
    _same(dev, ref)
    assert dev.fail.tolist()[:3] == [0, 1, 0] and dev.fail[3] == 1



# ---- the pair kind ------------------------------------------------------------------------------------------------
PAIR_CHAINS = [["RLI"], ["RLI", "MEGNO"], ["MEGNO", "RLI"]]


def _pairs(name, n=160):
    from chaos_b200 import pair_frame, pair_start
    sys, x0 = _system(name)
    x0 = x0[:n]
    if name == "wrapped":
        x0 = x0[:, :2]
    a = np.random.default_rng(41).uniform(0, 2 * np.pi, n)
    xis = np.stack([np.cos(a), np.sin(a)], axis=1)
    z0 = np.array([pair_start(sys, x, u, 1e-7 if name != "linear" else 1e-9)[0] for x, u in zip(x0, xis)])
    return sys, z0, np.array([pair_frame(u) for u in xis])


@pytest.mark.parametrize("members", PAIR_CHAINS, ids=",".join)
@pytest.mark.parametrize("name", ["standard", "wrapped", "linear"])
@pytest.mark.parametrize("tau", [1, 4])
def test_pair_indicator_matches_oracle(oracle, members, name, tau):
    from chaos_b200 import record_indicator_pairs
    sys, z0, W0 = _pairs(name)
    N = 200 if name != "linear" else 40
    grid = sorted({g for g in (tau, 2 * tau, 10 * tau, 25 * tau, N) if g <= N})
    ns = 2 * sys.s
    dev = record_indicator_pairs(sys, z0, W0, N, tau, members, grid, ns=ns)
    ref = oracle.oracle_indicator_pairs(sys, z0, W0, N, tau, members, grid, ns=ns)
    _same(dev, ref)


def test_pair_indicator_windows_and_failure(oracle):
    from chaos_b200 import record_indicator_pairs
    sys, z0, W0 = _pairs("standard", 64)
    W0[5, 2, 0] = 1e-3                      # pairing failure at the first handoff
    z0[9, 1] = np.inf                       # state failure
    grid = [8, 16, 40, 96, 200]
    dev = record_indicator_pairs(sys, z0, W0, 200, 4, ["RLI", "MEGNO"], grid, launch_steps=8)
    ref = oracle.oracle_indicator_pairs(sys, z0, W0, 200, 4, ["RLI", "MEGNO"], grid)
    _same(dev, ref)
    assert dev.fail[5] == 1 and dev.fail[9] == 1 and (np.delete(dev.fail, [5, 9]) == 0).all()
