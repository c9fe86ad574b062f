"""advance_ensemble on the B200 against the oracle, bit for bit, for table methods (leapfrogs, Kahan-Li 6 / 8, a
table with zero weights at both ends) and Gauss(3), the result of every orbit independent of the chunking, and a
failing Gauss orbit in the middle of the ensemble (test/integrator-catalog/ic_ac17_23.jl:36-60)."""
from __future__ import annotations

import numpy as np
import pytest

from chaos_b200 import (SABA, SABAC, SBAB, SBABC, CalvoSanzSerna4, Gauss, HenonHeilesFlow, KahanLi, Leapfrog, Ruth3, SplittingMethod,
                        SymplecticEuler, advance_ensemble, suzuki_jump)
from chaos_b200.systems import random_energy_starts
from helpers import same_bits

pytestmark = pytest.mark.gpu

FLOW = HenonHeilesFlow()
METHODS = {"DKD": Leapfrog("DKD"), "KDK": Leapfrog("KDK"), "KL6": KahanLi(6), "KL8": KahanLi(8),
           "KL7": KahanLi("s7odr6"), "SABA5": SABA(5), "SBAB4": SBAB(4), "Ruth3": Ruth3(),
           "CSS4": CalvoSanzSerna4(), "Suzuki8": suzuki_jump(Leapfrog(), 8), "SEKD": SymplecticEuler("KD"),
           "SABAC2": SABAC(2), "SBABC4": SBABC(4), "Gauss3": Gauss()}


def _starts(n=3000, seed=11):
    return np.asarray(random_energy_starts(0.125, n, seed))


@pytest.mark.parametrize("name", list(METHODS))
@pytest.mark.parametrize("n", [0, 1, 57])
def test_advance_matches_oracle(oracle, name, n):
    m = METHODS[name]
    x0 = _starts()
    s, ok = advance_ensemble(m, FLOW, x0, 0.05, n)
    rs, rok = oracle.oracle_advance(m, FLOW, x0, 0.05, n)
    assert same_bits(s, rs) and np.array_equal(ok, rok)


@pytest.mark.parametrize("name", ["KDK", "KL8", "Gauss3"])
def test_chunking_changes_no_bit(name):
    m = METHODS[name]
    x0 = _starts(2000, 12)
    a, oka = advance_ensemble(m, FLOW, x0, 0.05, 40)
    b, okb = advance_ensemble(m, FLOW, x0, 0.05, 40, chunk=7)
    c, okc = advance_ensemble(m, FLOW, x0, 0.05, 40, chunk=1000)
    assert same_bits(a, b) and same_bits(a, c) and (oka == okb).all() and (oka == okc).all()


def test_gauss_failure_in_the_ensemble(oracle):
    good = _starts(2, 5)
    x0 = np.array([good[0], [40.0, 40.0, 0.0, 0.0], good[1]])
    s, ok = advance_ensemble(Gauss(), FLOW, x0, 0.05, 10)
    rs, rok = oracle.oracle_advance(Gauss(), FLOW, x0, 0.05, 10)
    assert ok.tolist() == [True, False, True] and np.array_equal(ok, rok)
    assert same_bits(s, rs) and not np.isfinite(s[1]).any()


def test_custom_table(oracle):
    # a table with a zero drift first and a zero kick last: the pending kick crosses every step boundary
    m = SplittingMethod([0.0, 0.6, 0.4], [0.3, 0.7, 0.0], order=1, palindromic=False, name="custom")
    x0 = _starts(500, 13)
    s, ok = advance_ensemble(m, FLOW, x0, 0.03, 101)
    rs, rok = oracle.oracle_advance(m, FLOW, x0, 0.03, 101)
    assert same_bits(s, rs) and ok.all() and rok.all()
