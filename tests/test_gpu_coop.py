"""The cooperative lattice kernel (one orbit per group of d/2 lanes: sites spread over the lanes, the frame's columns
over the lanes at handoffs) against the oracle and against the one-thread kernel, bit for bit: open and ring
lattices of 2, 4 and 8 sites, per-orbit K and lengths, the escape stop, every register / unroll variant, Float64 and
mixed, and the failure records of a zero frame column and a non-finite start."""
from __future__ import annotations

import dataclasses

import numpy as np
import pytest

from chaos_b200 import HouseholderQR, QRSpectrum, StandardMapChain
from chaos_b200.ensemble import EnsembleClass, propagate_ensemble
from chaos_b200.propagate import FrameSpec
from helpers import same_bits, states_equal, uniform_starts

pytestmark = pytest.mark.gpu


def _chain_class(d, n, tau, seed, precision="fp64", escape=1e3, nmax=3000, ring=False, lanes=0, W0=None, x0=None):
    rng = np.random.default_rng(seed)
    k = min(d, 8)
    sysm = StandardMapChain(d // 2, 1.0, 0.05, boundary="ring" if ring else "open")
    x0 = uniform_starts(n, d, seed) if x0 is None else x0
    K = rng.uniform(0.5, 3.0, n)
    L = np.maximum(tau, (np.exp(rng.uniform(np.log(50), np.log(nmax), n)) // tau).astype(np.int64) * tau)
    if W0 is None:
        W0 = np.broadcast_to(np.eye(d)[:, :k], (n, d, k)).copy()
    return EnsembleClass(sysm, x0, FrameSpec(k, (QRSpectrum(HouseholderQR()),), W0), tau, int(nmax // tau * tau), K=K,
                         lengths=L, escape=escape, precision=precision, lanes=lanes)


def _same(a, b):
    return (np.array_equal(a.code, b.code) and np.array_equal(a.hstep, b.hstep) and same_bits(a.x, b.x)
            and same_bits(a.W, b.W) and states_equal(a.states, b.states))


@pytest.mark.parametrize("d,tau,ring", [(4, 10, False), (8, 10, False), (8, 10, True), (16, 20, False),
                                        (16, 20, True)])
@pytest.mark.parametrize("escape", [1e3, 25.0])
def test_coop_matches_oracle(oracle, d, tau, ring, escape):
    c = _chain_class(d, 333, tau, 300 + d, escape=escape, ring=ring, lanes=d // 2)
    dev = propagate_ensemble([c])[0]
    ref = oracle.oracle_ensemble(c.sys, c.x0, c.N, c.frame, tau=c.tau, K=c.K, lengths=c.lengths, escape=c.escape)
    assert np.array_equal(dev.code, ref["code"]) and np.array_equal(dev.hstep, ref["hstep"])
    assert same_bits(dev.x, ref["x"]) and same_bits(dev.W, ref["W"]) and states_equal(dev.states, ref["states"])


@pytest.mark.parametrize("d,tau", [(4, 10), (8, 10), (16, 20)])
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("minb,unroll", [(1, 1), (2, 0), (4, 1)])
def test_coop_equals_one_thread_kernel(d, tau, precision, minb, unroll):
    base = _chain_class(d, 290, tau, 40 + d, precision=precision, escape=30.0)
    one = propagate_ensemble([dataclasses.replace(base, lanes=1, minb=minb, unroll=unroll or tau)])[0]
    coop = propagate_ensemble([dataclasses.replace(base, lanes=d // 2, minb=minb, unroll=unroll or tau)])[0]
    assert _same(one, coop)


def test_coop_failure_records(oracle):
    d, n = 8, 96
    W0 = np.broadcast_to(np.eye(d), (n, d, d)).copy()
    W0[::3, :, 5] = 0.0                      # a zero column: QRSpectrum's pivot failure at the first handoff
    x0 = uniform_starts(n, d, 9)
    x0[1::7, 3] = np.nan                      # a non-finite start: the state failure
    c = _chain_class(d, n, 10, 9, W0=W0, x0=x0, lanes=4)
    dev = propagate_ensemble([c])[0]
    ref = oracle.oracle_ensemble(c.sys, c.x0, c.N, c.frame, tau=c.tau, K=c.K, lengths=c.lengths, escape=c.escape)
    assert (ref["code"] != 0).any() and np.array_equal(dev.code, ref["code"])
    assert np.array_equal(dev.hstep, ref["hstep"]) and same_bits(dev.W, ref["W"])
    assert states_equal(dev.states, ref["states"])
