"""The explicit table catalog (src/Integrators/tables.jl, tables_near.jl, splitting.jl): every constructor the
reference exports, checked the way test/integrator-catalog/ic_ac01_03.jl checks it, on the binary64 tables in exact
rational arithmetic (each double is a dyadic rational): the sum conditions, the palindromic symmetry, the digits, the
linear order of the step matrix of the harmonic oscillator (AC2), the triple-jump and Suzuki builders against their
closed forms and against an independent composition (AC3a), Yoshida's solution A against Kahan-Li s7odr6 and the
stage counts (AC3b), McLachlan's z and its error ratio (AC3b3), the Sofroniou-Spaletta print (AC3b4), the
Calvo-Sanz-Serna table against its RKN form (AC3b5), the force-evaluation counts (decision D113) and the adjoint."""
from __future__ import annotations

import math
from fractions import Fraction

import mpmath
import numpy as np
import pytest

import chaos_b200 as cb
from chaos_b200 import HenonHeilesFlow, IntegratorMap

EPS = 2.0 ** -52

# (id, constructor, nominal order, declared palindromic (None: not asserted), digits of the tabulated constants)
CATALOG = [
    ("S1DK", lambda: cb.SymplecticEuler("DK"), 1, False, math.inf),
    ("S1KD", lambda: cb.SymplecticEuler("KD"), 1, False, math.inf),
    ("S2DKD", lambda: cb.Leapfrog("DKD"), 2, True, math.inf),
    ("S2KDK", lambda: cb.Leapfrog("KDK"), 2, True, math.inf),
    ("S3", cb.McLachlan2, 2, True, math.inf),
    ("S4", cb.Ruth3, 3, False, math.inf),
    ("S5", cb.ForestRuth, 4, True, math.inf),
    ("S6-4", lambda: cb.triple_jump(cb.Leapfrog(), 4), 4, True, math.inf),
    ("S6-6", lambda: cb.triple_jump(cb.Leapfrog(), 6), 6, True, math.inf),
    ("S6-8", lambda: cb.triple_jump(cb.Leapfrog(), 8), 8, True, math.inf),
    ("S7-4", lambda: cb.suzuki_jump(cb.Leapfrog(), 4), 4, True, math.inf),
    ("S7-6", lambda: cb.suzuki_jump(cb.Leapfrog(), 6), 6, True, math.inf),
    ("S7-8", lambda: cb.suzuki_jump(cb.Leapfrog(), 8), 8, True, math.inf),
    ("S8", cb.PEFRL, 4, True, 16),
    ("S9", cb.CalvoSanzSerna4, 4, None, 18),
    ("S11-6A", lambda: cb.Yoshida(6, "A"), 6, True, 15),
    ("S11-8D", lambda: cb.Yoshida(8, "D"), 8, True, 15),
    ("S11-8A", lambda: cb.Yoshida(8, "A"), 8, True, 15),
    ("S12-6", lambda: cb.KahanLi(6), 6, True, 20),
    ("S12-8", lambda: cb.KahanLi(8), 8, True, 20),
    ("S12-s7odr6", lambda: cb.KahanLi("s7odr6"), 6, True, 20),
    ("S13", cb.SofroniouSpaletta10, 10, True, 32),
] + [(f"SABA{n}", (lambda n=n: cb.SABA(n)), 2, True, 40) for n in range(1, 5)] \
  + [(f"SBAB{n}", (lambda n=n: cb.SBAB(n)), 2, True, 40) for n in range(1, 5)] \
  + [("ABA864", cb.ABA864, 4, True, 40), ("ABAH864", cb.ABAH864, 4, True, 40)]
IDS = [c[0] for c in CATALOG]


def _kickpos(c, d):
    """Kick positions (the cumulative drift before each kick) and weights, zero kicks dropped, exactly."""
    acc, pos, w = Fraction(0), [], []
    for ci, di in zip(c, d):
        acc += Fraction(ci)
        if di != 0.0:
            pos.append(acc)
            w.append(Fraction(di))
    return pos, w


def _mat_mul(A, B):
    return [[A[0][0] * B[0][0] + A[0][1] * B[1][0], A[0][0] * B[0][1] + A[0][1] * B[1][1]],
            [A[1][0] * B[0][0] + A[1][1] * B[1][0], A[1][0] * B[0][1] + A[1][1] * B[1][1]]]


def _steppoly(c, d, deg, num=Fraction):
    """The step matrix of the oscillator q' = p, p' = -q as a matrix polynomial in tau truncated at `deg`:
    M = prod_i K_i D_i, D_i = I + c_i tau E12, K_i = I - d_i tau E21 (the first stage rightmost)."""
    zero, one = num(0), num(1)
    M = [[[one, zero], [zero, one]]] + [[[zero, zero], [zero, zero]] for _ in range(deg)]
    for ci, di in zip(c, d):
        for a, (r, s) in ((num(ci), (0, 1)), (-num(di), (1, 0))):
            if a == 0:
                continue
            new = [[row[:] for row in m] for m in M]
            for j in range(1, deg + 1):
                # (a X M_(j-1)): X = E_rs moves row s of M_(j-1) into row r
                for col in range(2):
                    new[j][r][col] += a * M[j - 1][s][col]
            M = new
    return M


def _rotpoly(deg, num=Fraction):
    out, P = [], [[num(1), num(0)], [num(0), num(1)]]
    A = [[num(0), num(1)], [num(-1), num(0)]]
    fact = 1
    for j in range(deg + 1):
        if j:
            fact *= j
        out.append([[P[r][s] / fact for s in range(2)] for r in range(2)])
        P = _mat_mul(P, A)
    return out


@pytest.mark.parametrize("mid,make,p,sym,dtab", CATALOG, ids=IDS)
def test_sum_conditions_symmetry_digits(mid, make, p, sym, dtab):
    """AC1 (ic_ac01_03.jl:14-47) on the binary64 tables."""
    m = make()
    c, d = cb.coefficients(m)
    k = len(c)
    assert len(d) == k and k >= 1 and cb.stage_count(m) == k
    et = max(EPS, 10.0 ** (-dtab))
    assert abs(float(sum(Fraction(v) for v in c) - 1)) <= 4 * k * et
    assert abs(float(sum(Fraction(v) for v in d) - 1)) <= 4 * k * et
    assert cb.table_digits(m) == dtab
    if sym is True:
        assert cb.is_palindromic(m)
        assert all(c[i] == c[k - 1 - i] for i in range(k))
        assert all(d[i] == d[k - 2 - i] for i in range(k - 1)) and d[k - 1] == 0.0
    elif sym is False:
        assert not cb.is_palindromic(m)
    src = [s.strip() for s in cb.method_source(m).split(",")]
    assert src and all(src)
    assert k <= 128 and IntegratorMap(m, HenonHeilesFlow(), 0.05).to_cl().n_stages == k


@pytest.mark.parametrize("mid,make,p,sym,dtab", CATALOG, ids=IDS)
def test_linear_order(mid, make, p, sym, dtab):
    """AC2 (ic_ac01_03.jl:50-66): the Taylor coefficients of the step matrix through the nominal order are those of
    the rotation, within 64 eps_tab S^p, S = 1 + sum |c| + sum |d|."""
    m = make()
    c, d = cb.coefficients(m)
    et = max(EPS, 10.0 ** (-dtab))
    S = 1 + sum(abs(v) for v in c) + sum(abs(v) for v in d)
    M, R = _steppoly(c, d, p + 1), _rotpoly(p + 1)
    dif = [max(abs(float(M[j][r][s] - R[j][r][s])) for r in range(2) for s in range(2)) for j in range(p + 2)]
    assert all(dif[j] <= 64 * et * S ** p for j in range(p + 1))
    assert cb.nominal_order(m) == p


def _leapfrog_composition_weights(order, suzuki):
    with mpmath.workprec(256):
        w, n = [mpmath.mpf(1)], 2
        while n < order:
            if suzuki:
                s = 1 / (4 - mpmath.power(4, mpmath.mpf(1) / (n + 1)))
                w = [s * x for x in w] * 2 + [(1 - 4 * s) * x for x in w] + [s * x for x in w] * 2
            else:
                z1 = 1 / (2 - mpmath.power(2, mpmath.mpf(1) / (n + 1)))
                w = [z1 * x for x in w] + [(1 - 2 * z1) * x for x in w] + [z1 * x for x in w]
            n += 2
        return w


def test_triple_jump_and_suzuki_closed_forms():
    """AC3a (ic_ac01_03.jl:69-98): the fourth-order triple jump and Forest-Ruth kick with theta, 1 - 2 theta, theta
    at theta / 2, 1/2, 1 - theta / 2; every level's kick count; the step polynomial equals the composition of leapfrog
    pieces with the 256-bit fractions; the binary64 triple jump 8 within 64 eps of the 256-bit one."""
    with mpmath.workprec(256):
        th = 1 / (2 - mpmath.cbrt(2))
        for m in (cb.triple_jump(cb.Leapfrog(), 4), cb.ForestRuth()):
            pos, w = _kickpos(*cb.coefficients(m))
            assert len(w) == 3
            assert max(abs(mpmath.mpf(float(x)) - y) for x, y in zip(w, (th, 1 - 2 * th, th))) <= 8 * EPS
            assert max(abs(mpmath.mpf(float(x)) - y) for x, y in zip(pos, (th / 2, mpmath.mpf(1) / 2, 1 - th / 2))) \
                <= 8 * EPS
    deg = 12
    for builder, suz, counts in ((cb.triple_jump, False, (3, 9, 27)), (cb.suzuki_jump, True, (5, 25, 125))):
        for order, cnt in zip((4, 6, 8), counts):
            m = builder(cb.Leapfrog(), order)
            c, d = cb.coefficients(m)
            assert sum(1 for v in d if v != 0.0) == cnt
            assert cb.nominal_order(m) == order
            wts = _leapfrog_composition_weights(order, suz)
            pos, w = _kickpos(c, d)
            # the composition of leapfrogs kicks with weight w_j at the middle of piece j
            with mpmath.workprec(256):
                acc, qpos = mpmath.mpf(0), []
                for x in wts:
                    qpos.append(acc + x / 2)
                    acc += x
                assert max(abs(mpmath.mpf(float(a)) - b) for a, b in zip(w, wts)) <= 64 * EPS
                assert max(abs(mpmath.mpf(float(a)) - b) for a, b in zip(pos, qpos)) <= 64 * EPS
            P = _steppoly(c, d, deg)
            with mpmath.workprec(256):
                Q = None
                lf = _steppoly((0.5, 0.5), (1.0, 0.0), deg, num=mpmath.mpf)
                for x in wts:
                    sc = [[[e * x ** j for e in row] for row in lf[j]] for j in range(deg + 1)]
                    Q = sc if Q is None else [
                        [[sum((sc[i][r][t] * Q[j - i][t][s] for i in range(j + 1) for t in range(2)), mpmath.mpf(0))
                          for s in range(2)] for r in range(2)] for j in range(deg + 1)]
                err = max(abs(mpmath.mpf(float(P[j][r][s])) - Q[j][r][s])
                          for j in range(deg + 1) for r in range(2) for s in range(2))
            assert err <= 1e-13


def test_yoshida_against_kahan_li_and_stage_counts():
    """AC3b (ic_ac01_03.jl:101-111): Yoshida 6A and Kahan-Li s7odr6 are independent prints of one method; Yoshida
    6A has 8 stages, 8A and 8D 16; Kahan-Li 6 and 8 kick 9 and 17 times."""
    pa, wa = _kickpos(*cb.coefficients(cb.Yoshida(6, "A")))
    pb, wb = _kickpos(*cb.coefficients(cb.KahanLi("s7odr6")))
    assert len(wa) == 7 and len(wb) == 7
    assert max(abs(float(x - y)) for x, y in zip(wa, wb)) <= 1e-14
    assert max(abs(float(x - y)) for x, y in zip(pa, pb)) <= 1e-14
    assert cb.stage_count(cb.Yoshida(6, "A")) == 8 and cb.stage_count(cb.Yoshida(8, "D")) == 16
    assert cb.stage_count(cb.Yoshida(8, "A")) == 16
    assert sum(1 for v in cb.KahanLi(6).d if v) == 9 and sum(1 for v in cb.KahanLi(8).d if v) == 17
    with pytest.raises(ValueError):
        cb.Yoshida(6, "D")


def test_mclachlan_z_and_error_ratio():
    """AC3b3 (ic_ac01_03.jl:113-136): z = 0.1932 of McLachlan's Table 2, kicks of 1/2 after the drifts z and 1 - z,
    and 4 ||E_S3|| / ||E_leapfrog|| < 0.5 for the tau^3 coefficient of the oscillator's step matrix."""
    m = cb.McLachlan2()
    c, d = cb.coefficients(m)
    with mpmath.workprec(256):
        y = mpmath.cbrt(2 * mpmath.sqrt(326) - 36)
        z = (y ** 2 + 6 * y - 2) / (12 * y)
        assert abs(float(z) - 0.1932) <= 5e-5
        pos, w = _kickpos(c, d)
        assert len(w) == 2 and all(x == Fraction(1, 2) for x in w)
        assert max(abs(mpmath.mpf(float(a)) - b) for a, b in zip(pos, (z, 1 - z))) <= 64 * EPS
    R = _rotpoly(3)

    def E(mm):
        P = _steppoly(*cb.coefficients(mm), 3)
        return np.linalg.norm(np.array([[float(P[3][r][s] - R[3][r][s]) for s in range(2)] for r in range(2)]), 2)
    ratio = 4 * E(m) / E(cb.Leapfrog("DKD"))
    assert ratio < 0.5 and abs(ratio - 0.318) < 0.01


def test_sofroniou_spaletta_print():
    """AC3b4 (ic_ac01_03.jl:138-155): 32 digits, 35 kicks, the Table 1 norm sum |d| = 6.18133."""
    m = cb.SofroniouSpaletta10()
    c, d = cb.coefficients(m)
    assert cb.table_digits(m) == 32 and sum(1 for v in d if v) == 35 and cb.stage_count(m) == 36
    assert abs(sum(abs(v) for v in d) - 6.18133) <= 1e-5


def _hh_force(q):
    return np.array([-q[0] - 2 * q[0] * q[1], -q[1] - q[0] * q[0] + q[1] * q[1]])


def test_calvo_sanz_serna_rkn_form(oracle):
    """AC3b5 (ic_ac01_03.jl:154-185): the table (kick first, gamma_1 = 0, sum b = 1, gamma_5 = 1) and one step of the
    splitting on the oracle against the RKN formulas Q_i = q + h gamma_i p + h^2 sum_(j<i) b_j (gamma_i - gamma_j)
    f(Q_j), here on the Henon-Heiles flow, within 16 eps max(1, |z|)."""
    m = cb.CalvoSanzSerna4()
    c, d = cb.coefficients(m)
    assert cb.table_digits(m) == 18 and len(c) == 5 and c[0] == 0.0
    et = max(EPS, 1e-18)
    gam = np.cumsum(c)
    assert abs(sum(d) - 1) <= 4 * et * 5 and abs(gam[4] - 1) <= 4 * et * 5
    rng = np.random.default_rng(20261012 + 41000 + 40 * 3 + 1)
    z0 = rng.uniform(-0.5, 0.5, (20, 4))
    h = 0.1
    a, ok = oracle.oracle_advance(m, HenonHeilesFlow(), z0, h, 1)
    assert ok.all()
    for zi, ai in zip(z0, a):
        q, p = zi[:2], zi[2:]
        F = []
        for i in range(5):
            Q = q + h * gam[i] * p
            for j in range(i):
                Q = Q + h * h * d[j] * (gam[i] - gam[j]) * F[j]
            F.append(_hh_force(Q))
        pn = p + h * sum(d[i] * F[i] for i in range(5))
        qn = q + h * p + h * h * sum(d[i] * (1 - gam[i]) * F[i] for i in range(5))
        assert np.max(np.abs(ai - np.concatenate([qn, pn]))) <= 16 * EPS * max(1.0, np.max(np.abs(zi)))


def _expected_evals(c, d):
    """Force evaluations of one step: adjacent kicks with no drift between them share one (ic_helpers.jl:134-144)."""
    cnt, prev = 0, -1
    for i, di in enumerate(d):
        if di == 0.0:
            continue
        merged = prev >= 0 and all(v == 0.0 for v in c[prev + 1:i + 1])
        if not merged:
            cnt += 1
        prev = i
    return cnt


def _expected_cyclic(c, d):
    """Per step of a long run: maximal runs of kicks in the cyclic drift/kick sequence (ic_helpers.jl:147-156)."""
    ev = []
    for ci, di in zip(c, d):
        if ci != 0.0:
            ev.append("D")
        if di != 0.0:
            ev.append("K")
    if "D" not in ev:
        return 1 if "K" in ev else 0
    return sum(1 for i in range(len(ev)) if ev[i] == "K" and ev[i - 1] != "K")


@pytest.mark.parametrize("mid,make,p,sym,dtab", CATALOG, ids=IDS)
def test_force_evaluations(mid, make, p, sym, dtab):
    """Decision D113 (splitting.jl:62-97): the isolated count and the long-run count against an independent count."""
    m = make()
    c, d = cb.coefficients(m)
    assert cb.isolated_force_evaluations(m) == _expected_evals(c, d)
    assert cb.force_evaluations(m) == _expected_cyclic(c, d)


def test_leapfrog_kdk_costs_one_evaluation_per_step():
    m = cb.Leapfrog("KDK")
    assert cb.isolated_force_evaluations(m) == 2 and cb.force_evaluations(m) == 1


def test_adjoint(oracle):
    """adjoint_method (splitting.jl:125-133): symmetric tables are their own adjoint, the adjoint of DK is KD, and
    S*(-tau) after S(tau) returns the start to round-off on the oracle."""
    kl = cb.KahanLi(8)
    assert cb.adjoint_method(kl) is kl
    kd = cb.adjoint_method(cb.SymplecticEuler("DK"))
    assert kd.c == cb.SymplecticEuler("KD").c and kd.d == cb.SymplecticEuler("KD").d
    assert cb.method_name(kd) == "symplectic Euler DK (adjoint)"
    rng = np.random.default_rng(5)
    z0 = rng.uniform(-0.4, 0.4, (16, 4))
    for m in (cb.SymplecticEuler("DK"), cb.Ruth3(), cb.CalvoSanzSerna4()):
        adj = cb.adjoint_method(m)
        assert not adj.palindromic and cb.nominal_order(adj) == cb.nominal_order(m)
        z1, ok1 = oracle.oracle_advance(m, HenonHeilesFlow(), z0, 0.1, 1)
        z2, ok2 = oracle.oracle_advance(adj, HenonHeilesFlow(), z1, -0.1, 1)
        assert ok1.all() and ok2.all() and np.max(np.abs(z2 - z0)) <= 64 * EPS
        # the method itself does not invert the step: S(-tau) S(tau) = id + O(tau^(p+1)), far above round-off
        z3, _ = oracle.oracle_advance(m, HenonHeilesFlow(), z1, -0.1, 1)
        assert np.max(np.abs(z3 - z0)) > 1e4 * EPS


def test_corrected_methods():
    """SABAC / SBABC (tables_near.jl:100-128): the corrector coefficients of Table II (closed forms in binary64 for
    the small n), the names and orders, and the record an IntegratorMap of the Henon-Heiles flow hands the kernel."""
    with mpmath.workprec(200):
        exact = {("SABA", 1): mpmath.mpf(1) / 12, ("SABA", 2): (2 - mpmath.sqrt(3)) / 24,
                 ("SABA", 3): (54 - 13 * mpmath.sqrt(15)) / 648, ("SBAB", 1): -mpmath.mpf(1) / 24,
                 ("SBAB", 2): mpmath.mpf(1) / 72, ("SBAB", 3): (13 - 5 * mpmath.sqrt(5)) / 288,
                 ("SBAB", 4): (3861 - 791 * mpmath.sqrt(21)) / 64800}
        for (kind, n), v in exact.items():
            m = (cb.SABAC if kind == "SABA" else cb.SBABC)(n)
            assert abs(mpmath.mpf(m.c) - v) <= 1e-14 * abs(v)
            assert cb.method_name(m) == f"{kind}C{n}" and cb.nominal_order(m) == (4 if n >= 2 else 2)
    assert cb.SABAC(4).c == float("0.003396775048208601331532157783492144")
    mc = cb.SABAC(2)
    assert cb.is_palindromic(cb.SBABC(5)) and cb.adjoint_method(mc) is mc
    assert cb.force_evaluations(cb.SABAC(2)) == cb.isolated_force_evaluations(cb.SABA(2)) + 2
    with pytest.raises(ValueError):
        cb.SABAC(11)
    cs = IntegratorMap(cb.SABAC(2), HenonHeilesFlow(), 0.1).to_cl()
    assert cs.corrector == 1 and cs.eps == cb.SABAC(2).c and cs.n_stages == cb.SABA(2).stages


def test_pow_is_not_near_a_tie():
    """The binary64 powers the builders use (2^(1/3), 2^(1/5), 2^(1/7), 4^(1/3), 4^(1/5), 4^(1/7), McLachlan's
    cube root) are rounded once from 200 bits; each lies at least 1e-3 ulp from a rounding tie, so any pow accurate
    to 0.5 + 1e-3 ulp (Julia's double-double evaluation among them) returns the same double."""
    cases = [(2.0, 1.0 / 3.0), (2.0, 1.0 / 5.0), (2.0, 1.0 / 7.0), (4.0, 1.0 / 3.0), (4.0, 1.0 / 5.0),
             (4.0, 1.0 / 7.0), (2.0 * math.sqrt(326.0) - 36.0, 1.0 / 3.0)]
    from chaos_b200.systems import _pow
    for x, y in cases:
        with mpmath.workprec(200):
            v = mpmath.power(mpmath.mpf(x), mpmath.mpf(y))
            r = _pow(x, y)
            ulp = math.ulp(r)
            frac = abs((v - mpmath.mpf(r)) / ulp)
        assert frac <= 0.5 and 0.5 - frac >= 1e-3
        assert r == x ** y          # the platform's pow agrees


@pytest.mark.parametrize("make", [lambda: cb.SABAC(2), lambda: cb.SBABC(3), lambda: cb.SABAC(5)], ids=["SABAC2", "SBABC3", "SABAC5"])
def test_corrected_method_on_the_oracle(oracle, make):
    """The corrected step on the Henon-Heiles flow (stepper.jl:142-160): symmetric, S(-tau) S(tau) = id to
    round-off; its tangent (the corrector Jacobians around the base table's) equals central differences of the
    forward step; and it differs from the base table's step by the corrector's O(tau^3) kicks."""
    m = make()
    flow = HenonHeilesFlow()
    rng = np.random.default_rng(8)
    z0 = rng.uniform(-0.3, 0.3, (12, 4))
    z1, ok1 = oracle.oracle_advance(m, flow, z0, 0.1, 1)
    z2, ok2 = oracle.oracle_advance(m, flow, z1, -0.1, 1)
    assert ok1.all() and ok2.all() and np.max(np.abs(z2 - z0)) <= 64 * EPS
    zb, _ = oracle.oracle_advance(m.base, flow, z0, 0.1, 1)
    diff = np.max(np.abs(zb - z1))
    assert 1e-9 < diff < 1e-2
    from chaos_b200.propagate import FrameSpec
    sysm = IntegratorMap(m, flow, 0.1)
    h = 1e-6
    for z in z0[:4]:
        # the one-step Jacobian: W after one step from W0 = I with a non-replacing chain (Benettin would normalise)
        r = oracle.oracle_frames(sysm, z[None], 1, [FrameSpec(4, (), np.eye(4)[None])], tau=1, math="portable")[0]
        T = r["W"][0]
        fd = np.empty((4, 4))
        for j in range(4):
            e = np.zeros(4)
            e[j] = h
            zp, _ = oracle.oracle_advance(m, flow, (z + e)[None], 0.1, 1)
            zm, _ = oracle.oracle_advance(m, flow, (z - e)[None], 0.1, 1)
            fd[:, j] = (zp[0] - zm[0]) / (2 * h)
        assert np.max(np.abs(T - fd)) <= 1e-8
