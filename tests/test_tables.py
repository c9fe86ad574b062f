"""The near-integrable tables SABA_n and SBAB_n (src/Integrators/tables_near.jl:1-73), built here from the
Gauss-Legendre and Gauss-Lobatto rules in 330-bit arithmetic and rounded once: SABA_1 and SBAB_1 are the DKD and KDK
leapfrogs, SABA_2 and SBAB_2 their closed forms, and every table's kicks are a quadrature of the free flight exact for
the monomials of degree <= 2n - 1 and not of degree 2n (the moment statement of
test/integrator-catalog/ic_ac04_08.jl:67-83, here on the Float64 tables in exact rational arithmetic)."""
from __future__ import annotations

from fractions import Fraction

import mpmath
import numpy as np
import pytest

from chaos_b200 import SABA, SBAB, HenonHeilesFlow, Leapfrog
from chaos_b200.systems import random_energy_starts

EPS = Fraction(1, 2 ** 52)


def test_first_rows_are_the_leapfrogs():
    assert SABA(1).c == Leapfrog("DKD").c and SABA(1).d == Leapfrog("DKD").d
    assert SBAB(1).c == Leapfrog("KDK").c and SBAB(1).d == Leapfrog("KDK").d


def test_second_rows_closed_forms():
    with mpmath.workprec(200):
        a = float(mpmath.mpf(1) / 2 - mpmath.sqrt(3) / 6)
        b = float(mpmath.sqrt(3) / 3)
    assert SABA(2).c == (a, b, a) and SABA(2).d == (0.5, 0.5, 0.0)
    assert SBAB(2).c == (0.0, 0.5, 0.5, 0.0) and SBAB(2).d == (1 / 6, 2 / 3, 1 / 6, 0.0)


@pytest.mark.parametrize("n", range(1, 11))
@pytest.mark.parametrize("make", [SABA, SBAB], ids=["SABA", "SBAB"])
def test_kicks_are_a_quadrature_of_degree_2n_minus_1(make, n):
    m = make(n)
    assert m.palindromic and m.stages == (n + 1 if make is SABA else n + 2)
    pos, acc = [], Fraction(0)
    w = []
    for c, d in zip(m.c, m.d):
        acc += Fraction(c)
        if d != 0.0:
            pos.append(acc)
            w.append(Fraction(d))

    def mom(k):
        return abs(sum(wi * p ** k for wi, p in zip(w, pos)) - Fraction(1, k + 1))
    assert max(mom(k) for k in range(2 * n)) <= 64 * EPS
    assert mom(2 * n) > Fraction(1, 10 ** 14)


def test_saba_keeps_the_energy(oracle):
    flow = HenonHeilesFlow()
    x0 = np.asarray(random_energy_starts(0.125, 20, 9))
    for m in (SABA(3), SBAB(3)):
        states, ok = oracle.oracle_advance(m, flow, x0, 0.05, 2000)
        H0 = np.array([flow.hamiltonian(z) for z in x0])
        H1 = np.array([flow.hamiltonian(z) for z in states])
        assert ok.all() and np.max(np.abs(H1 - H0)) <= 1e-3
