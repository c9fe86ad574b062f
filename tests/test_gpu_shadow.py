"""The two-trajectory estimator on the B200 against the oracle, bit for bit: every end record (reference and shadow
states, the Neumaier sum, d_prev, code, step, value) for the lifted and wrapped standard maps, the Froeschle map, a
ring lattice, a linear map and the Henon-Heiles integrator maps; seeded and given directions; launch windows;
the failure records and the lowest failing orbit's error."""
from __future__ import annotations

import numpy as np
import pytest

from chaos_b200 import (FroeschleMap, Gauss, HenonHeilesFlow, IntegratorMap, KahanLi, LinearSymplecticMap,
                        NumericalHealthError, StandardMap, StandardMapChain, WrappedStandardMap, propagate_shadow,
                        random_energy_starts, torus_state)
from helpers import uniform_starts

pytestmark = pytest.mark.gpu


def _cases():
    rng = np.random.default_rng(21)
    std = uniform_starts(300, 2, 22)
    return {
        "standard": (StandardMap(6.0), std, 600, 1),
        "standard_tau5": (StandardMap(1.2), std, 600, 5),
        "wrapped": (WrappedStandardMap(6.0), np.array([torus_state(z) for z in std]), 600, 1),
        "froeschle": (FroeschleMap(1.5, 1.5, 0.05), uniform_starts(300, 4, 23), 500, 10),
        "ring": (StandardMapChain(4, 1.0, 0.05, boundary="ring"), uniform_starts(200, 8, 24), 400, 10),
        # from the origin (AC1's start): elsewhere the cat map's growth soon puts d0 below the states' rounding
        "linear": (LinearSymplecticMap([[2.0, 1.0], [1.0, 1.0]]), np.zeros((100, 2)), 60, 3),
        "gauss": (IntegratorMap(Gauss(3, tol=1e-14), HenonHeilesFlow(), 0.01), random_energy_starts(1 / 8, 64, 25), 200, 10),
        "split": (IntegratorMap(KahanLi(8), HenonHeilesFlow(), 0.05), random_energy_starts(1 / 8, 128, 26), 400, 10),
    }


@pytest.mark.parametrize("name", list(_cases()))
@pytest.mark.parametrize("given", [False, True])
def test_shadow_matches_oracle(oracle, name, given):
    sys, x0, N, tau = _cases()[name]
    U0 = np.random.default_rng(7).normal(size=(len(x0), sys.d)) if given else None
    d0 = 1e-8
    dev = propagate_shadow(sys, x0, N, d0=d0, tau=tau, seed=9, U0=U0)
    u = None
    if given:   # the host normalises U0 by safe_norm; hand the oracle the same unit vectors
        from chaos_b200.shadow import _safe_norm
        u = np.array([[v / _safe_norm(row) for v in row] for row in U0])
    ref = oracle.oracle_shadow(sys, x0, N, d0=d0, tau=tau, seed=9, U0=u)
    assert dev.states.tobytes() == ref.tobytes()
    X2 = np.array([f[0]["X2"] for f in dev.finals])
    assert np.all(np.isfinite(X2))


def test_shadow_launch_windows_and_chunks(oracle):
    sys, x0, N, tau = _cases()["froeschle"]
    a = propagate_shadow(sys, x0, N, d0=1e-9, tau=tau, seed=3)
    b = propagate_shadow(sys, x0, N, d0=1e-9, tau=tau, seed=3, launch_steps=30, chunk=77)
    assert a.states.tobytes() == b.states.tobytes()


def test_shadow_failures(oracle):
    """A non-finite start has a non-finite start separation: Algorithm 1 fails it with "separation" (code 2) at
    step 0; an orbit that overflows later fails with "state" (code 1) at its handoff; a wrapped start whose seeded
    separation folds (d0 > pi) fails with "separation" against d0 (code 3). The lowest failing orbit is reported,
    and every record equals the oracle's."""
    sys, x0, N, tau = _cases()["standard_tau5"]
    x = x0[:50].copy()
    x[17, 0] = np.nan
    x[31, 1] = 1e308          # overflows to inf inside the first handoff's five steps
    with pytest.raises(NumericalHealthError) as ei:
        propagate_shadow(sys, x, N, d0=1e-8, tau=tau, seed=1)
    ref = oracle.oracle_shadow(sys, x, N, d0=1e-8, tau=tau, seed=1)
    bad = np.flatnonzero(ref["code"] != 0)
    assert list(bad) == [17, 31] and list(ref["code"][bad]) == [2, 1]
    assert ei.value.orbit == 18 and ei.value.what == "separation" and ei.value.step == 0
    with pytest.raises(NumericalHealthError) as ei:
        propagate_shadow(sys, x[18:], N, d0=1e-8, tau=tau, seed=1)
    ref2 = oracle.oracle_shadow(sys, x[18:], N, d0=1e-8, tau=tau, seed=1)
    j = int(np.flatnonzero(ref2["code"] != 0)[0])
    assert ei.value.what == "state" and ei.value.orbit == j + 1 and ei.value.step == ref2["step"][j]
    xw = np.array([torus_state([1.0, 0.2])] * 8)
    with pytest.raises(NumericalHealthError) as ei:
        propagate_shadow(WrappedStandardMap(0.5), xw, 10, d0=5.0, seed=2)
    ref = oracle.oracle_shadow(WrappedStandardMap(0.5), xw, 10, d0=5.0, seed=2)
    first = int(np.flatnonzero(ref["code"] != 0)[0])
    assert ei.value.what == "separation" and ei.value.step == 0 and ei.value.orbit == first + 1
