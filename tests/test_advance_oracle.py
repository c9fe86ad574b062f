"""advance_ensemble on the oracle (CPU), src/Integrators/ensemble.jl:1-45: against the pinned single steps of the
IntegratorMap oracle where the reference's advance_n merges nothing across a step (DKD tables, Gauss), the merged
kick of KDK at the rounding level, energy kept by the symplectic tables, the failing Gauss orbit all NaN with the
others untouched (the AC18 statements of test/integrator-catalog/ic_ac17_23.jl:36-60), and the host-side checks."""
from __future__ import annotations

import numpy as np
import pytest

from chaos_b200 import Gauss, HenonHeilesFlow, KahanLi, Leapfrog, advance_ensemble
from chaos_b200.systems import random_energy_starts

FLOW = HenonHeilesFlow()


def _starts(n=40, seed=3):
    return np.asarray(random_energy_starts(0.125, n, seed))


def _single_steps(oracle, m, x0, tau, n):
    out = np.array(x0, dtype=np.float64)
    T = np.empty(16)
    for j in range(len(out)):
        z = out[j].copy()
        for _ in range(n):
            if isinstance(m, Gauss):
                oracle.lib().oracle_gauss3_step(oracle._dp(z), tau, m.maxiter, np.nan if m.tol is None else m.tol,
                                                oracle._dp(T))
            else:
                c = np.ascontiguousarray(m.c, dtype=np.float64)
                d = np.ascontiguousarray(m.d, dtype=np.float64)
                oracle.lib().oracle_split_step(oracle._dp(z), tau, m.stages, oracle._dp(c), oracle._dp(d),
                                               oracle._dp(T))
        out[j] = z
    return out


@pytest.mark.parametrize("m", [Leapfrog("DKD"), KahanLi(6), KahanLi(8), Gauss()], ids=["DKD", "KL6", "KL8", "Gauss3"])
def test_no_merge_across_steps_equals_single_steps(oracle, m):
    x0 = _starts()
    states, ok = oracle.oracle_advance(m, FLOW, x0, 0.05, 60)
    assert ok.all()
    assert states.tobytes() == _single_steps(oracle, m, x0, 0.05, 60).tobytes()


def test_kdk_merges_the_boundary_kicks(oracle):
    x0 = _starts()
    m = Leapfrog("KDK")
    states, ok = oracle.oracle_advance(m, FLOW, x0, 0.05, 200)
    single = _single_steps(oracle, m, x0, 0.05, 200)
    assert ok.all()
    assert np.max(np.abs(states - single)) <= 1e-12
    assert not np.array_equal(states, single)          # one kick of weight 1 is not two kicks of 1/2 in Float64


@pytest.mark.parametrize("m,bound", [(KahanLi(8), 1e-11), (Leapfrog("DKD"), 5e-4)], ids=["KL8", "DKD"])
def test_symplectic_tables_keep_the_energy(oracle, m, bound):
    x0 = _starts(30, 4)
    states, ok = oracle.oracle_advance(m, FLOW, x0, 0.05, 2000)
    H0 = np.array([FLOW.hamiltonian(z) for z in x0])
    H1 = np.array([FLOW.hamiltonian(z) for z in states])
    assert ok.all() and np.max(np.abs(H1 - H0)) <= bound


def test_gauss_failure_is_all_nan_and_isolated(oracle):
    good = _starts(2, 5)
    bad = np.array([40.0, 40.0, 0.0, 0.0])               # the fixed point diverges at this distance
    x0 = np.array([good[0], bad, good[1]])
    states, ok = oracle.oracle_advance(Gauss(), FLOW, x0, 0.05, 10)
    assert ok.tolist() == [True, False, True]
    assert not np.isfinite(states[1]).any()
    ref, _ = oracle.oracle_advance(Gauss(), FLOW, good, 0.05, 10)
    assert states[[0, 2]].tobytes() == ref.tobytes()


def test_host_checks():
    with pytest.raises(TypeError):
        advance_ensemble(KahanLi(6), object(), np.zeros((2, 4)), 0.05, 3)
    with pytest.raises(ValueError):
        advance_ensemble(KahanLi(6), FLOW, np.zeros((2, 3)), 0.05, 3)
