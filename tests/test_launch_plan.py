"""The device launch plan of `propagate` (src/Tangent/propagate.jl:146-193) and its hooks: the reference's own
known answers for the budget (test/tangent-core/tc_d44.jl:205-213), the plan and the launches per chunk, and on the
GPU the relaunch that the plan and the `_before_launch` hook drive, bit for bit the one-launch run."""
import math

import numpy as np
import pytest

from chaos_b200 import launch_plan as LP


def _budget_L(ns, tau):   # the definition, independently: the largest multiple of tau with ns 1e-9 L 1024 <= 1
    m = 0
    while ns * 1e-9 * ((m + 1) * tau) * 1024 <= 1.0:
        m += 1
    return m * tau


def test_budget_known_answers():
    assert LP.budget_steps(25.0, 1) == 39062 and LP.budget_steps(25.0, 10) == 39060
    assert LP.budget_steps(100.0, 1) == 9765 and LP.budget_steps(100.0, 10) == 9760
    assert LP.budget_steps(97657.0, 10) == 0   # just above 1 / (10 x 1024 x 1e-9) = 97656.25
    assert isinstance(LP.budget_steps(25.0, 1), int)
    for ns in (3.0, 20.2, 25.0, 100.0, 5000.0):
        for tau in (1, 2, 10):
            assert LP.budget_steps(ns, tau) == _budget_L(ns, tau)
    assert LP.DEFAULT_GPU_NS == 100.0 and LP.LAUNCH_WAVE == 1024 and LP.LAUNCH_BUDGET_S == 1.0


def test_plan():
    # N = 1e6 with the record 25 ns: 26 launches per chunk (tc_d44.jl:233-239), the estimate within the budget
    for tau in (1, 10):
        L, cap = LP.device_plan(None, 1_000_000, tau, 25.0)
        assert L == (39062 if tau == 1 else 39060) and LP.launches(1_000_000, L) == 26
        assert 25.0 * 1e-9 * L * max(cap, 1024) <= 1.0 + 1e-9
    assert LP.device_plan(None, 100, 10, 97657.0) == (0, 0)
    assert LP.device_plan(None, 50, 10, 25.0)[0] == 50                       # never above N
    assert LP.device_plan(70, 1000, 10, 25.0) == (70, max(1024, LP.budget_orbits(25.0, 70)))   # forced keeps the floor
    assert LP.launches(100, 0) == 0 and LP.launches(100, 30) == 4
    LP.LAUNCH_STEPS = 7
    try:
        with pytest.raises(ValueError):
            LP.forced_launch(2)
        assert LP.forced_launch(7) == 7
    finally:
        LP.LAUNCH_STEPS = None


@pytest.mark.gpu
def test_hook_and_relaunch():
    """With the hook set, propagate runs each chunk launch by launch from the host (the forced L = 70 here), calls the
    hook before every launch with the chunk and launch indices and the live carried buffers, and the result is the
    one-launch run's bit for bit; the one-wave record exists after the first call."""
    from chaos_b200 import FroeschleMap, HouseholderQR, QRSpectrum, propagate
    from helpers import identity_frames, same_bits, states_equal, uniform_starts
    n, N, tau = 300, 500, 10
    x0 = uniform_starts(n, 4, seed=4)
    sysm = FroeschleMap(1.5, 1.5, 0.05)
    kw = dict(k=4, tau=tau, reducers=(QRSpectrum(HouseholderQR()),), W0=identity_frames(n, 4, 4), finals=False)
    full = propagate(sysm, x0, N, **kw)
    assert full.provenance["launches_per_chunk"] == 1 and full.provenance["launch_steps"] == N
    assert LP.gpu_step_ns("fp64", measure=False) is not None
    calls = []
    LP.BEFORE_LAUNCH = lambda dev, ci, li, carried: calls.append((ci, li, carried["x"].shape))
    LP.LAUNCH_STEPS = 70
    try:
        r = propagate(sysm, x0, N, chunk=128, **kw)
    finally:
        LP.BEFORE_LAUNCH = None
        LP.LAUNCH_STEPS = None
    assert same_bits(r.x, full.x) and same_bits(r.W, full.W) and states_equal(r.states, full.states)
    per = math.ceil(N / 70)
    assert r.provenance["launch_steps"] == 70 and r.provenance["launches_per_chunk"] == per
    assert [(c, l) for c, l, _ in calls] == [(c, l) for c in (1, 2, 3) for l in range(1, per + 1)]
    assert calls[0][2] == (128, 4) and calls[-1][2] == (n - 256, 4)
