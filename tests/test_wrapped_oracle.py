"""The torus forms of the coupled maps on the oracle (WrappedFroeschleMap, src/Systems/froeschle_map.jl:60-126, and
WrappedStandardMapChain, src/Systems/wrapped_standard_map_chain.jl), pinned by the reference's known answers:
the known point of torus_state and the lift round trip (test/coupled-maps/cm_ac05_06.jl:95-111), the count-overflow
construction that must give NaN in every component (cm_ac05_06.jl:140-166), the decoupled chain equal bit for bit to
independent wrapped standard maps (the decoupled limit of cm_ac07_12.jl:183 on the torus), and the wrapped orbit
lifting onto the lifted map's orbit."""
from __future__ import annotations

import math

import numpy as np
import pytest

from chaos_b200 import (MGS, Benettin, FroeschleMap, QRSpectrum, StandardMapChain, WrappedFroeschleMap,
                        WrappedStandardMap, WrappedStandardMapChain, lift, torus_state)
from chaos_b200.propagate import FrameSpec
from helpers import identity_frames, same_bits

EPS = 2.0 ** -52
LIM = 2.0 ** 53


def _run(oracle, sysm, x0, N, k=1, chain=None, tau=1):
    chain = chain or (Benettin(),)
    fr = [FrameSpec(k, chain, identity_frames(len(x0), sysm.d, k))]
    return oracle.oracle_frames(sysm, np.asarray(x0, dtype=np.float64), N, fr, tau=tau, math="portable")[0]


def test_known_torus_point():
    s = torus_state(WrappedFroeschleMap(0.5, 0.1, 1.0e-3), np.array([7.0, 0.5, -1.0, 0.25]))
    assert len(s) == 8
    assert s[4] == 1 and s[6] == -1 and s[5] == 0 and s[7] == 0
    assert abs(s[0] - (7.0 - 2 * math.pi)) <= 4 * math.ulp(7.0)   # Julia's eps(7.0)


@pytest.mark.parametrize("sysm", [WrappedFroeschleMap(0.5, 0.1, 1.0e-3), WrappedStandardMapChain(2, 3.0, 0.2),
                                  WrappedStandardMapChain(5, 1.0, 0.6102, boundary="ring")], ids=repr)
def test_torus_round_trip(sysm):
    rng = np.random.default_rng(11)
    d = sysm.d
    for _ in range(20):
        z = rng.uniform(-100, 100, d)
        s = torus_state(sysm, z)
        assert len(s) == 2 * d
        assert all(0 <= s[j] < 2 * math.pi for j in range(d))
        assert all(s[d + j] == round(s[d + j]) for j in range(d))
        assert np.all(np.abs(lift(sysm, s) - z) <= 16 * math.ulp(100.0))


def test_count_overflow_gives_nan(oracle):
    """cm_ac05_06.jl:140-166: a count that reaches maxintfloat poisons the state; one below stays finite."""
    w0 = WrappedFroeschleMap(0.0, 0.0, 0.0)
    r = _run(oracle, w0, [[6.0, 0.0, 3.0, 0.0, LIM - 1, 0.0, 0.0, 0.0], [6.0, 0.0, 3.0, 0.0, LIM - 2, 0.0, 0.0, 0.0]], 1)
    assert np.isnan(r["x"][0]).all() and r["code"][0] == 1
    assert np.isfinite(r["x"][1]).all() and r["x"][1][4] == LIM - 1 and r["code"][1] == 0
    w1 = WrappedFroeschleMap(-6.0, 0.0, 0.0)
    x1 = math.pi / 2 - 1
    r = _run(oracle, w1, [[x1, 0.0, 1.0, 0.0, 0.0, 0.0, LIM - 1, 0.0], [x1, 0.0, 1.0, 0.0, 0.0, 0.0, LIM - 2, 0.0]], 1)
    assert np.isnan(r["x"][0]).all() and np.isfinite(r["x"][1]).all() and r["x"][1][6] == LIM - 1
    wc0 = WrappedStandardMapChain(2, 0.0, 0.0)
    r = _run(oracle, wc0, [[6.0, 0.0, 3.0, 0.0, LIM - 1, 0.0, 0.0, 0.0], [6.0, 0.0, 3.0, 0.0, LIM - 2, 0.0, 0.0, 0.0]], 1)
    assert np.isnan(r["x"][0]).all() and np.isfinite(r["x"][1]).all() and r["x"][1][4] == LIM - 1
    wc1 = WrappedStandardMapChain(2, 6.0, 0.0)
    r = _run(oracle, wc1, [[math.pi / 2, 0.0, 1.0, 0.0, 0.0, 0.0, LIM - 1, 0.0],
                           [math.pi / 2, 0.0, 1.0, 0.0, 0.0, 0.0, LIM - 2, 0.0]], 1)
    assert np.isnan(r["x"][0]).all() and np.isfinite(r["x"][1]).all() and r["x"][1][6] == LIM - 1


@pytest.mark.parametrize("N", [2, 3, 5])
def test_decoupled_chain_is_independent_wrapped_maps(oracle, N):
    """eps = 0: every site of the wrapped chain is a WrappedStandardMap, bit for bit (state layout permuted)."""
    rng = np.random.default_rng(20 + N)
    n = 16
    z = rng.uniform(-20, 20, (n, 2 * N))
    chain = WrappedStandardMapChain(N, 2.5, 0.0)
    s0 = np.array([torus_state(chain, v) for v in z])
    rc = _run(oracle, chain, s0, 300)
    for j in range(N):
        site = np.array([[v[j], v[N + j], v[2 * N + j], v[3 * N + j]] for v in s0])
        rs = _run(oracle, WrappedStandardMap(2.5), site, 300)
        got = np.stack([rc["x"][:, j], rc["x"][:, N + j], rc["x"][:, 2 * N + j], rc["x"][:, 3 * N + j]], axis=1)
        assert same_bits(got, rs["x"])


@pytest.mark.parametrize("wrapped,lifted", [
    (WrappedFroeschleMap(0.5, 0.1, 1.0e-3), FroeschleMap(0.5, 0.1, 1.0e-3)),
    (WrappedStandardMapChain(3, 0.02, 0.01), StandardMapChain(3, 0.02, 0.01)),
    (WrappedStandardMapChain(4, 0.02, 0.01, boundary="ring"), StandardMapChain(4, 0.02, 0.01, boundary="ring"))],
    ids=repr)
def test_wrapped_orbit_lifts_onto_the_lifted_orbit(oracle, wrapped, lifted):
    """Regular orbits (small kicks): lift(s_n) follows z_n to the round-off of the lifted coordinates (which grow
    linearly, ulp ~1e-13 at 1000), and the exponent sums agree to 1e-9."""
    rng = np.random.default_rng(5)
    n, d = 24, wrapped.d
    z = rng.uniform(0, 2 * math.pi, (n, d))
    s0 = np.array([torus_state(wrapped, v) for v in z])
    rw = _run(oracle, wrapped, s0, 200, k=d, chain=(QRSpectrum(MGS()),), tau=5)
    rl = _run(oracle, lifted, z, 200, k=d, chain=(QRSpectrum(MGS()),), tau=5)
    back = np.array([lift(wrapped, v) for v in rw["x"]])
    assert np.max(np.abs(back - rl["x"]) / np.maximum(1.0, np.abs(rl["x"]))) <= 1e-9
    sw = rw["states"]["r0"]["sums"] if "sums" in rw["states"]["r0"].dtype.names else None
    if sw is not None:
        sl = rl["states"]["r0"]["sums"]
        assert np.max(np.abs(sw - sl)) <= 1e-9
