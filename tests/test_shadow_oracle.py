"""The two-trajectory estimator's oracle against the reference's analytic cases (test/lyap-two-trajectory/
l2_analytic.jl AC1 to AC4) and the host API's argument checks. CPU only."""
from __future__ import annotations

import math

import numpy as np
import pytest

from chaos_b200 import LinearSymplecticMap, StandardMap, WrappedStandardMap, torus_state


def _nX2(e):
    return e["sum_s"] + e["sum_c"]


@pytest.mark.parametrize("tau", [1, 5, 10])
@pytest.mark.parametrize("n", [20, 100, 1000])
def test_ac1_linear_map_at_origin(oracle, tau, n):
    """AC1: the cat map A = [[2, 1], [1, 1]] from the origin, u0 = (1, 0), d0 = 2^-20: n X2 = ln ||A^n u0|| =
    ln sqrt(F_{2n+1}^2 + F_{2n}^2) (Fibonacci numbers, exact in integers)."""
    if n % tau:
        pytest.skip("n must be a multiple of tau")
    sys = LinearSymplecticMap([[2.0, 1.0], [1.0, 1.0]])
    ends = oracle.oracle_shadow(sys, np.zeros((1, 2)), n, d0=2.0 ** -20, tau=tau, U0=[[1.0, 0.0]])
    f = [0, 1]
    while len(f) < 2 * n + 2:
        f.append(f[-1] + f[-2])
    exact = 0.5 * math.log(f[2 * n + 1] ** 2 + f[2 * n] ** 2)
    assert ends["code"][0] == 0 and ends["step"][0] == n
    assert abs(_nX2(ends[0]) - exact) <= 1e-13 * n * (1 + tau)


@pytest.mark.parametrize("tau", [1, 10])
def test_ac2_shear_at_origin(oracle, tau):
    """AC2: StandardMap(K = 0) at the origin with u0 = (cos t, sin t): n X2 = ln sqrt((a + n b)^2 + b^2)."""
    th = np.random.default_rng(2).uniform(0, 2 * np.pi, 20)
    U0 = np.stack([np.cos(th), np.sin(th)], axis=1)
    n = 1000
    ends = oracle.oracle_shadow(StandardMap(0.0), np.zeros((20, 2)), n, d0=2.0 ** -20, tau=tau, U0=U0)
    for j in range(20):
        a, b = U0[j]
        exact = math.log(math.hypot(a + n * b, b) / math.hypot(a, b))
        assert abs(_nX2(ends[j]) - exact) <= 1e-11


def test_ac3_hyperbolic_fixed_point(oracle):
    """AC3: the standard map's hyperbolic fixed point (0, 0), K = 2, tau = 1, small d0: n X2 approaches
    n ln mu_+ + ln(|c_1| ||v_u||) (the unstable eigenvalue mu_+ and the start's component along it)."""
    K, n, d0 = 2.0, 100, 1e-9
    th = np.random.default_rng(3).uniform(0, 2 * np.pi, 50)
    U0 = np.stack([np.cos(th), np.sin(th)], axis=1)
    ends = oracle.oracle_shadow(StandardMap(K), np.zeros((50, 2)), n, d0=d0, tau=1, U0=U0)
    s = math.sqrt(K * (K + 4))
    mu = (2 + K + s) / 2
    vu = math.sqrt(1 + ((s - K) / 2) ** 2)
    for j in range(50):
        c1 = abs(U0[j, 0] * (K + s) / 2 + U0[j, 1]) / s
        exact = n * math.log(mu) + math.log(c1 * vu)
        if c1 > 1e-3:   # far from the stable direction: the asymptotic form holds within the nonlinearity
            assert abs(_nX2(ends[j]) - exact) <= 1e-6 * n


def test_ac4_minimal_image(oracle):
    """AC4: the wrapped map at K = 0, p = 0: a pair straddling x = 0 reads n X2 = 0 like the same pair at x = 1
    (the separation is the minimal image), and the mirror case across p = 0 with u0 = (0, 1) reads ln sqrt(n^2 + 1)."""
    d0, n = 2.0 ** -20, 1000
    sys = WrappedStandardMap(0.0)
    strad, plain = torus_state([-d0 / 2, 0.0]), torus_state([1.0, 0.0])
    ends = oracle.oracle_shadow(sys, np.array([strad, plain]), n, d0=d0, tau=1, U0=[[1.0, 0.0], [1.0, 0.0]])
    assert (ends["code"] == 0).all()
    assert abs(_nX2(ends[0])) <= 1e-12 and abs(_nX2(ends[1])) <= 1e-12
    assert abs(_nX2(ends[0]) - _nX2(ends[1])) <= 1e-12
    mirror = torus_state([1.0, -d0 / 2])
    e = oracle.oracle_shadow(sys, np.array([mirror]), n, d0=d0, tau=1, U0=[[0.0, 1.0]])
    e_ro = 2.0 ** -52 * 2 * math.pi / d0          # the round-off of a wrapped coordinate relative to d0
    assert abs(_nX2(e[0]) - 0.5 * math.log(n * n + 1)) <= 2 * n * e_ro


@pytest.mark.parametrize("L", [6, 30, 600])
def test_launch_windows_carry_bitwise(oracle, L):
    """A run split into launch windows (D44) equals the one-window run bit for bit."""
    x0 = np.random.default_rng(4).uniform(0, 2 * np.pi, (40, 2))
    a = oracle.oracle_shadow(StandardMap(6.0), x0, 600, d0=1e-8, tau=3, seed=5)
    b = oracle.oracle_shadow(StandardMap(6.0), x0, 600, d0=1e-8, tau=3, seed=5, launch_steps=L)
    assert a.tobytes() == b.tobytes()


def test_argument_errors():
    """The reference's ArgumentErrors (ValueError here): d0, N / tau, U0 length, chunk; and Algorithm 1's start
    check (a realised separation outside [d0/2, 2 d0] raises before any launch)."""
    from chaos_b200 import NumericalHealthError, propagate_shadow
    x0 = np.zeros((2, 2))
    with pytest.raises(ValueError, match="d0"):
        propagate_shadow(StandardMap(1.0), x0, 10, d0=-1.0, seed=1)
    with pytest.raises(ValueError, match="multiple of tau"):
        propagate_shadow(StandardMap(1.0), x0, 10, d0=1e-8, tau=3, seed=1)
    with pytest.raises(ValueError, match="one vector per orbit"):
        propagate_shadow(StandardMap(1.0), x0, 10, d0=1e-8, seed=1, U0=[[1.0, 0.0]])
    with pytest.raises(ValueError, match="chunk"):
        propagate_shadow(StandardMap(1.0), x0, 10, d0=1e-8, seed=1, chunk=0)
    # wrapped map, d0 = 5 > pi: the minimal image folds the start separation to 2 pi - 5 < d0 / 2
    x = np.array([torus_state([1.0, 0.0])])
    with pytest.raises(NumericalHealthError) as ei:
        propagate_shadow(WrappedStandardMap(0.5), x, 10, d0=5.0, seed=1, U0=[[1.0, 0.0]])
    assert ei.value.what == "separation" and ei.value.step == 0 and ei.value.threshold == 5.0


@pytest.mark.parametrize("mk", [lambda: __import__("chaos_b200").WrappedFroeschleMap(1.5, 1.5, 0.05),
                                lambda: __import__("chaos_b200").WrappedStandardMapChain(3, 1.0, 0.05)],
                         ids=["wrapped-froeschle", "wrapped-chain"])
def test_wrapped_coupled_maps_dimension_mismatch(mk):
    """On the wrapped coupled maps the reference's start check (two_trajectory.jl:158-162) evaluates the generic
    `displaced(sys, x, d0 u0) = x + d0 u0` (separation.jl:17) with an s-vector state and a d-vector direction
    (s = 8 against d = 4; s = 4N against d = 2N) and StaticArrays throws DimensionMismatch before any launch: the
    host side raises the same error, seeded directions or given ones."""
    from chaos_b200 import propagate_shadow
    from chaos_b200.foundation import DimensionMismatch
    sysm = mk()
    x0 = np.array([sysm.torus_state(z) for z in np.random.default_rng(1).uniform(0, 6, (3, sysm.d))])
    with pytest.raises(DimensionMismatch):
        propagate_shadow(sysm, x0, 100, d0=1e-8, tau=10, seed=1)
    with pytest.raises(DimensionMismatch):
        propagate_shadow(sysm, x0, 100, d0=1e-8, tau=10, U0=np.ones((3, sysm.d)))
