"""The oracle pinned against the reference's own known-answer tests (CPU only).

Each test replays a criterion of the reference's suite on the oracle (the restatement the GPU kernels are then
compared with bit for bit): closed forms and bitwise identities that hold whatever the last bit of sin / cos / log,
so they pin the restated algorithm itself. Sources are cited per test.
"""
from __future__ import annotations

import math
from decimal import Decimal, getcontext
from fractions import Fraction

import numpy as np
import pytest

from chaos_b200 import (CGS, FLI, GALI, MEGNO, MGS, RGS, SALI, AugmentedQR, Benettin, FroeschleMap, GivensQR,
                        HouseholderQR, LinearSymplecticMap, QRSpectrum, StandardMap, StandardMapChain)
from chaos_b200.propagate import FrameSpec
from helpers import haar_frames, identity_frames, same_bits, states_equal, uniform_starts

EPS = 2.0 ** -52
ALGS = [CGS(), MGS(), RGS(), HouseholderQR(), AugmentedQR(), GivensQR()]
getcontext().prec = 60


def _one(oracle, sys, x0, N, k, reducers, W0, tau=1, math_="portable", **kw):
    return oracle.oracle_frames(sys, np.atleast_2d(x0), N, [FrameSpec(k, tuple(reducers), W0)], tau=tau,
                                math=math_, **kw)[0]


def _final(r, reducers, i=0, d=2):
    st = r["states"][i]
    out = []
    for j, red in enumerate(reducers):
        out.append(red.final(st[f"r{j}"], d) if isinstance(red, GALI) else red.final(st[f"r{j}"]))
    return out


def test_fibonacci_exact(oracle):
    """W_n = A^n and x_n = A^n x0 bitwise for A = [[2,1],[1,1]], n = 1..35 (test/tangent-core/tc_ac01_04.jl:4-17)."""
    A = np.array([[2.0, 1.0], [1.0, 1.0]])
    x0 = np.array([3.0, 5.0])
    for n in range(1, 36):
        r = _one(oracle, LinearSymplecticMap(A), x0, n, 2, (), identity_frames(1, 2, 2))
        An = np.linalg.matrix_power(A.astype(object), n).astype(float)
        assert np.array_equal(r["W"][0], An)
        assert np.array_equal(r["x"][0], An @ x0)


@pytest.mark.parametrize("tau", [1, 5, 10])
def test_linear_renormalisation(oracle, tau):
    """S_n + ln||w_n|| = ln||A^n w0|| to 8 n eps and S_n / n -> ln((3 + sqrt 5)/2) within 2e-3 at n = 1e4
    (tc_ac01_04.jl:19-50), with the one-vector Benettin reducer."""
    N = 10_000
    A = np.array([[2.0, 1.0], [1.0, 1.0]])
    m = 20
    W0 = haar_frames(m, 2, 1, 5)
    r = oracle.oracle_frames(LinearSymplecticMap(A), np.zeros((m, 2)), N, [FrameSpec(1, (Benettin(),), W0)], tau=tau)[0]
    M = [[2, 1], [1, 1]]
    P = [[1, 0], [0, 1]]
    e = N
    base = M
    while e:   # exact integer power
        if e & 1:
            P = [[P[0][0] * base[0][0] + P[0][1] * base[1][0], P[0][0] * base[0][1] + P[0][1] * base[1][1]],
                 [P[1][0] * base[0][0] + P[1][1] * base[1][0], P[1][0] * base[0][1] + P[1][1] * base[1][1]]]
        base = [[base[0][0] * base[0][0] + base[0][1] * base[1][0], base[0][0] * base[0][1] + base[0][1] * base[1][1]],
                [base[1][0] * base[0][0] + base[1][1] * base[1][0], base[1][0] * base[0][1] + base[1][1] * base[1][1]]]
        e >>= 1
    lam = math.log((3 + math.sqrt(5)) / 2)
    for j in range(m):
        w = [Fraction(float(W0[j, 0, 0])), Fraction(float(W0[j, 1, 0]))]
        y0 = P[0][0] * w[0] + P[0][1] * w[1]
        y1 = P[1][0] * w[0] + P[1][1] * w[1]
        ref = (Decimal(y0.numerator) / Decimal(y0.denominator)) ** 2 + (Decimal(y1.numerator) / Decimal(y1.denominator)) ** 2
        ref = float(ref.ln() / 2)
        st = r["states"][j]["r0"]
        S = st["sum_s"] + st["sum_c"]
        assert abs(S + math.log(np.linalg.norm(r["W"][j])) - ref) <= 8 * N * EPS
        assert abs(S / N - lam) <= 2e-3
        assert int(st["n"]) == N


def test_standard_map_K0_shear(oracle):
    """K = 0: W_n = [[1, n], [0, 1]] and x_n = x0 + n p0 bitwise (tc_ac01_04.jl:52-64)."""
    for n in (1, 10, 1000, 10 ** 6):
        r = _one(oracle, StandardMap(0.0), [0.25, 0.5], n, 2, (), identity_frames(1, 2, 2))
        assert np.array_equal(r["W"][0], np.array([[1.0, n], [0.0, 1.0]]))
        assert np.array_equal(r["x"][0], np.array([0.25 + 0.5 * n, 0.5]))


@pytest.mark.parametrize("alg", ALGS, ids=repr)
def test_qr_K0_closed_form(oracle, alg):
    """GS AC2 / HH AC4(b): Q_0 = (e_2, e_1), K = 0: S_1 = (1/2) ln(n^2 + 1) to 8 n eps, S_2 = -S_1 to 8 n eps
    (test/lyap-gram-schmidt/gs_ac01_05.jl:27-47, test/lyap-householder-qr/hh_exact.jl:3-33)."""
    W0 = np.array([[[0.0, 1.0], [1.0, 0.0]]])
    for n in (1, 10, 1000, 10 ** 4):
        r = _one(oracle, StandardMap(0.0), [0.3, 0.7], n, 2, (QRSpectrum(alg),), W0)
        f = QRSpectrum(alg).final(r["states"][0]["r0"])
        S = f["sum"] + f["comp"]
        ref = float((Decimal(n) ** 2 + 1).ln() / 2)
        assert abs(S[0] - ref) <= 8 * n * EPS
        assert abs(S[1] + S[0]) <= 8 * n * EPS
        if n == 10 ** 4:
            assert f["lambda"][0] <= math.log(1e4) / 1e4 + 1e-12


@pytest.mark.parametrize("alg", ALGS, ids=repr)
def test_shear_exact(oracle, alg):
    """HH AC4(a): the shear [[1,1],[0,1]] from W_0 = I keeps Q = I and every sum exactly 0 for 1e4 handoffs
    (hh_exact.jl:3-16)."""
    r = _one(oracle, LinearSymplecticMap(np.array([[1.0, 1.0], [0.0, 1.0]])), [0.0, 0.0], 10_000, 2,
             (QRSpectrum(alg),), identity_frames(1, 2, 2))
    f = QRSpectrum(alg).final(r["states"][0]["r0"])
    assert np.all(f["sum"] == 0) and np.all(f["comp"] == 0) and np.all(f["lambda"] == 0)
    assert np.array_equal(r["W"][0], np.eye(2))


@pytest.mark.parametrize("alg", ALGS, ids=repr)
@pytest.mark.parametrize("tau", [1, 2, 5])
def test_cat_map_spectrum(oracle, alg, tau):
    """HH AC5 (hh_exact.jl:36-70): the cat map A = [[2,1],[1,1]] at its fixed point from Q_0 = I:
    |lambda_1 - ln mu - ln(c)/n| to rounding and lambda_1 + lambda_2 = 0 to rounding, mu = (3 + sqrt 5)/2."""
    n = 1000
    r = _one(oracle, LinearSymplecticMap(np.array([[2.0, 1.0], [1.0, 1.0]])), [0.0, 0.0], n, 2, (QRSpectrum(alg),),
             identity_frames(1, 2, 2), tau=tau)
    f = QRSpectrum(alg).final(r["states"][0]["r0"])
    mu = (Decimal(3) + Decimal(5).sqrt()) / 2
    c = 1 / (1 + ((Decimal(5).sqrt() - 1) / 2) ** 2).sqrt()
    expect = float(mu.ln() + c.ln() / n)
    assert abs(f["lambda"][0] - expect) <= 1e-12
    assert abs(f["lambda"][0] + f["lambda"][1]) <= 1e-13


@pytest.mark.parametrize("K", [0.5, 2 * math.pi, 10.0])
def test_cross_estimator_sums_bitwise(oracle, K):
    """MEGNO AC7(a) (test/megno/mg_ac06_08.jl:47-100): on the identical orbit the log sums of MEGNO, FLI and SALI
    are bitwise equal, and equal to one-vector Benettin runs per column."""
    m, N = 20, 2000
    x0 = uniform_starts(m, 2, 3)
    W0 = haar_frames(m, 2, 2, 4)
    chain = (MEGNO(replace=False), FLI(replace=False), SALI())
    r = _one(oracle, StandardMap(K), x0, N, 2, chain, W0)
    l1 = [_one(oracle, StandardMap(K), x0, N, 1, (Benettin(),), W0[:, :, i:i + 1]) for i in range(2)]
    for j in range(m):
        ms, fs, ss = _final(r, chain, j)
        assert np.array_equal(ms["sum"], fs["sum"]) and np.array_equal(ms["comp"], fs["comp"])
        assert np.array_equal(ms["sum"], ss["sum"]) and np.array_equal(ms["comp"], ss["comp"])
        for i in range(2):
            b = Benettin().final(l1[i]["states"][j]["r0"])
            assert ms["sum"][i] + ms["comp"][i] == b["sum"][0] + b["comp"][0]


def test_gali_columns_equal_sali(oracle):
    """GALI_4 columns 1-2 are bitwise a SALI k = 2 run on the same orbit and W0 (test/gali/ga_ac05_08.jl:356-397);
    the fused chain (GALI, SALI) gives that SALI record."""
    m, N = 32, 3000
    x0 = uniform_starts(m, 4, 6)
    W0 = haar_frames(m, 4, 4, 7)
    sysm = FroeschleMap(1.5, 1.5, 0.05)
    g = oracle.oracle_frames(sysm, x0, N, [FrameSpec(4, (GALI(), SALI()), W0)], tau=10)[0]
    s = oracle.oracle_frames(sysm, x0, N, [FrameSpec(2, (SALI(),), W0[:, :, :2])], tau=10)[0]
    assert same_bits(g["W"][:, :, :2], s["W"])
    for j in range(m):
        gs = g["states"][j]
        assert gs["r0"]["s"][0] == s["states"][j]["r0"]["s1_s"] and gs["r0"]["c"][1] == s["states"][j]["r0"]["s2_c"]
        assert same_bits(np.array([gs["r1"]["sali"]]), np.array([s["states"][j]["r0"]["sali"]]))


def test_megno_K0_closed_form(oracle):
    """MEGNO AC2 (test/megno/mg_ac01_05.jl:141-200): K = 0 shear from W_0 = I, tau = 1: column 1 has Y = Ybar =
    Ybar20 = 0 exactly; column 2 Y(n) = ln(n^2 + 1) - (1/n) sum_{i<n} ln(i^2 + 1) to 6 B_S(n)."""
    for n in (10, 100, 1000):
        r = _one(oracle, StandardMap(0.0), [0.4, 0.1], n, 2, (MEGNO(),), identity_frames(1, 2, 2))
        f = MEGNO().final(r["states"][0]["r0"])
        assert f["Y"][0] == 0 and f["Ybar"][0] == 0 and f["Ybar20"][0] == 0
        lp = sum((Decimal(i) ** 2 + 1).ln() for i in range(n))
        Ycf = float((Decimal(n) ** 2 + 1).ln() - lp / n)
        assert abs(f["Y"][1] - Ycf) <= 6 * 8 * EPS * (n + 4)


def test_chain_decoupled_equals_standard_map(oracle):
    """eps = 0: each site of the chain is a standard map, bitwise (test/coupled-maps/cm_ac07_12.jl:183)."""
    m, N, K = 16, 2000, 1.3
    q, p = uniform_starts(m, 4, 8), uniform_starts(m, 4, 88)
    r = _one(oracle, StandardMapChain(4, K, 0.0), np.hstack([q, p]), N, 2, (), haar_frames(m, 8, 2, 9))
    for j in range(4):
        s = _one(oracle, StandardMap(K), np.stack([q[:, j], p[:, j]], axis=1), N, 1, (), identity_frames(m, 2, 1))
        assert np.array_equal(r["x"][:, j], s["x"][:, 0]) and np.array_equal(r["x"][:, 4 + j], s["x"][:, 1])


@pytest.mark.parametrize("math_", ["libm", "portable"])
def test_readme_value_band(oracle, math_):
    """README.md:19-22: StandardMap(6), x0 = (0.1, 0.2), N = 1e5, k = 2, tau = 1, QRSpectrum(MGS()) gives
    lambda = +-1.1348588476487835 from a StableRNGs seeded frame (not reproducible here): a sanity band on
    lambda_1 and the exact pairing lambda_1 + lambda_2 = 0 to 1e-12."""
    r = _one(oracle, StandardMap(6.0), [0.1, 0.2], 100_000, 2, (QRSpectrum(MGS()),), haar_frames(1, 2, 2, 1),
             math_=math_)
    lam = QRSpectrum(MGS()).final(r["states"][0]["r0"])["lambda"]
    assert abs(lam[0] - 1.1348588476487835) <= 2e-2
    assert abs(lam[0] + lam[1]) <= 1e-12


def test_thread_count_and_relaunch_invariance(oracle):
    """propagate on the CPU equals a serial map of propagate_orbit bitwise for any chunk and thread count, and
    the step-chunked relaunch carries the state exactly (src/Tangent/propagate.jl:272-273, D44)."""
    m, N = 97, 1500
    x0 = uniform_starts(m, 4, 10)
    fr = [FrameSpec(4, (QRSpectrum(HouseholderQR()),), haar_frames(m, 4, 4, 11)), FrameSpec(2, (MEGNO(),), haar_frames(m, 4, 2, 12))]
    a = oracle.oracle_frames(FroeschleMap(1.5, 1.5, 0.05), x0, N, fr, tau=10, threads=1)
    b = oracle.oracle_frames(FroeschleMap(1.5, 1.5, 0.05), x0, N, fr, tau=10, threads=8)
    c = oracle.oracle_frames(FroeschleMap(1.5, 1.5, 0.05), x0, N, fr, tau=10, launch_steps=70)
    for f in range(2):
        for o in (b, c):
            assert same_bits(a[f]["W"], o[f]["W"]) and states_equal(a[f]["states"], o[f]["states"])
            assert same_bits(a[f]["x"], o[f]["x"])


def test_henon_heiles_saddle_tangent(oracle):
    """Hénon-Heiles tangent of one Gauss-3 step at the saddle S0 = (0, 1), p = 0 equals the exact linear flow:
    cos / sin (sqrt 3 t) in (q1, p1) and cosh / sinh (t) in (q2, p2) to 1e-9 (test/henon-heiles/hh_ac13_17.jl:64-83)."""
    h = 0.01
    z, T = oracle.gauss3_step(np.array([0.0, 1.0, 0.0, 0.0]), h, 50, 1e-14)
    assert np.allclose(z, [0.0, 1.0, 0.0, 0.0], atol=1e-15)
    w = math.sqrt(3.0)
    ex = np.zeros((4, 4))
    ex[0, 0] = ex[2, 2] = math.cos(w * h)
    ex[0, 2] = math.sin(w * h) / w
    ex[2, 0] = -w * math.sin(w * h)
    ex[1, 1] = ex[3, 3] = math.cosh(h)
    ex[1, 3] = math.sinh(h)
    ex[3, 1] = math.sinh(h)
    assert np.max(np.abs(T - ex)) <= 1e-9


def test_gauss3_order_and_symplecticity(oracle):
    """Gauss-3 (order 6): halving the step divides the one-step local error by about 2^7, and the step's
    Jacobian is symplectic (M' J M = J) to rounding (gauss.jl:176-192)."""
    z0 = np.array([0.0, 0.1, math.sqrt(2 * (1 / 8 - 0.1 ** 2 / 2 + 0.1 ** 3 / 3 - 0.05 ** 2 / 2)), 0.05])

    def flow(z, h, n):
        for _ in range(n):
            z, T = oracle.gauss3_step(z, h, 50, 1e-14)
        return z

    ref = flow(z0, 0.1 / 64, 64)
    e1 = np.max(np.abs(flow(z0, 0.1, 1) - ref))
    e2 = np.max(np.abs(flow(z0, 0.05, 2) - ref))
    assert 40 < e1 / e2 < 200
    _, T = oracle.gauss3_step(z0, 0.01, 50, 1e-14)
    J = np.block([[np.zeros((2, 2)), np.eye(2)], [-np.eye(2), np.zeros((2, 2))]])
    assert np.max(np.abs(T.T @ J @ T - J)) <= 1e-13


def test_ensemble_orbit_is_a_reference_call(oracle):
    """Each orbit of a batched uneven ensemble equals the reference call propagate_orbit(sys(K_i), x0_i, W0_i, N_i')
    with N_i' its own length, or the escape handoff (code 4) when max |p| passes the bound first."""
    rng = np.random.default_rng(3)
    n, tau = 40, 5
    x0 = uniform_starts(n, 2, 12)
    K = rng.uniform(0.5, 3.0, n)
    L = (rng.integers(1, 400, n) * tau).astype(np.int64)
    W0 = identity_frames(n, 2, 2)
    fr = FrameSpec(2, (QRSpectrum(HouseholderQR()),), W0)
    ens = oracle.oracle_ensemble(StandardMap(1.0), x0, int(L.max()), fr, tau=tau, K=K, lengths=L, escape=50.0)
    assert (ens["code"] == 4).any() and (ens["code"] == 0).any()
    for i in range(n):
        Ni = int(ens["hstep"][i])
        assert Ni == L[i] or ens["code"][i] == 4
        one = _one(oracle, StandardMap(float(K[i])), x0[i], Ni, 2, (QRSpectrum(HouseholderQR()),), W0[i:i + 1], tau=tau)
        assert same_bits(one["W"][0], ens["W"][i]) and same_bits(one["x"][0], ens["x"][i])
        assert states_equal(one["states"][:1], ens["states"][i:i + 1])
        if ens["code"][i] == 4:
            assert np.max(np.abs(ens["x"][i][1:])) > 50.0


# ---- table methods on the Henon-Heiles flow (src/Integrators/stepper.jl, tables.jl; test/henon-heiles) -------------
def _hh_starts(n, seed):
    from chaos_b200 import random_energy_starts
    return random_energy_starts(1 / 8, n, seed=seed)


def test_kahanli_table_shapes():
    """KahanLi(Float64, 8) is the palindromic composition of 17 leapfrogs (18 stages, the last kick weight zero);
    both sums are 1 to rounding; Leapfrog(:DKD) is (1/2, 1/2 | 1, 0)."""
    from chaos_b200 import KahanLi, Leapfrog
    m = KahanLi(8)
    assert m.stages == 18 and m.d[-1] == 0.0 and m.order == 8
    assert abs(sum(m.c) - 1) < 1e-14 and abs(sum(m.d) - 1) < 1e-14
    assert m.c == m.c[::-1] and m.d[:-1] == m.d[-2::-1]
    assert KahanLi(6).stages == 10 and KahanLi("s7odr6").stages == 8
    lf = Leapfrog("DKD")
    assert lf.c == (0.5, 0.5) and lf.d == (1.0, 0.0)


def test_split_step_commutes_with_reflection(oracle):
    """hh_ac01_05.jl AC3b: one KahanLi-8 step commutes with q1 -> -q1, p1 -> -p1 bit for bit (1000 random states)."""
    from chaos_b200 import KahanLi
    m = KahanLi(8)
    rng = np.random.default_rng(33)
    flip = np.array([-1.0, 1.0, -1.0, 1.0])
    for _ in range(1000):
        z = 2 * rng.random(4) - 1
        a, _ = oracle.split_step(z, 0.05, m)
        b, _ = oracle.split_step(z * flip, 0.05, m)
        assert np.array_equal(a * flip, b)


def test_split_energy_conservation(oracle):
    """hh_ac06_09.jl AC6: KahanLi-8 at tau = 1/20 keeps |H - H0| <= 1e-8 along E = 1/8 orbits (no drift)."""
    from chaos_b200 import HenonHeilesFlow, KahanLi
    m = KahanLi(8)
    H = HenonHeilesFlow.hamiltonian
    worst = 0.0
    for z0 in _hh_starts(4, 6):
        z, H0 = z0.copy(), H(z0)
        for _ in range(2000):
            z, _ = oracle.split_step(z, 1 / 20, m)
            worst = max(worst, abs(H(z) - H0))
    assert worst <= 1e-8


def test_split_time_reversal(oracle):
    """hh_ac01_05.jl AC3d: n steps, p -> -p, n steps, p -> -p returns to the start (regular E = 1/20 orbits)."""
    from chaos_b200 import KahanLi, Leapfrog, random_energy_starts
    flipp = np.array([1.0, 1.0, -1.0, -1.0])
    for m in (KahanLi(8), Leapfrog("DKD")):
        for z0 in random_energy_starts(1 / 20, 3, seed=8):
            z = z0.copy()
            for _ in range(2000):
                z, _ = oracle.split_step(z, 0.05, m)
            z = z * flipp
            for _ in range(2000):
                z, _ = oracle.split_step(z, 0.05, m)
            assert np.max(np.abs(z * flipp - z0)) <= 1e-11


def test_split_tangent_is_the_step_jacobian(oracle):
    """tangent_advance (stepper.jl:108-118): the tangent is symplectic (T' Omega T = Omega to rounding) and equals
    central differences of the step."""
    from chaos_b200 import KahanLi
    m = KahanLi(8)
    Om = np.block([[np.zeros((2, 2)), np.eye(2)], [-np.eye(2), np.zeros((2, 2))]])
    for z0 in _hh_starts(3, 9):
        _, T = oracle.split_step(z0, 0.05, m)
        assert np.max(np.abs(T.T @ Om @ T - Om)) <= 1e-14
        e = 1e-6
        fd = np.column_stack([(oracle.split_step(z0 + e * np.eye(4)[j], 0.05, m)[0] -
                               oracle.split_step(z0 - e * np.eye(4)[j], 0.05, m)[0]) / (2 * e) for j in range(4)])
        assert np.max(np.abs(T - fd)) <= 1e-8
