"""The recorder's oracle (CPU): a row at a grid step holds the finals of the same estimator run directly to that step
(src/Experiments/run_record.jl:1-3, R2), the monitor's residuals stay at the rounding level for the symplectic maps,
the running maxima are monotone, and splitting the run into launches changes no bit."""
from __future__ import annotations

import numpy as np
import pytest

from chaos_b200 import MGS, Benettin, HouseholderQR, QRSpectrum, StandardMap, WrappedStandardMap, torus_state
from chaos_b200.propagate import FrameSpec


def _starts(n, seed, wrapped=False):
    z = np.random.default_rng(seed).uniform(0, 2 * np.pi, (n, 2))
    return np.array([torus_state(v) for v in z]) if wrapped else z


@pytest.mark.parametrize("est", [QRSpectrum(MGS()), QRSpectrum(HouseholderQR()), Benettin()], ids=repr)
@pytest.mark.parametrize("wrapped", [False, True])
def test_rows_are_the_direct_runs_finals(oracle, est, wrapped):
    sys = WrappedStandardMap(1.3) if wrapped else StandardMap(1.3)
    x0 = _starts(24, 5, wrapped)
    tau, grid = 5, [10, 50, 200, 500]
    rec = oracle.oracle_record(sys, x0, 500, tau, est, grid)
    k = 1 if isinstance(est, Benettin) else 2
    assert (rec["fail"] == 0).all()
    for g, N in enumerate(grid):
        W0 = np.broadcast_to(np.eye(2)[:, :k], (24, 2, k)).copy()
        ref = oracle.oracle_frames(sys, x0, N, [FrameSpec(k, (est,), W0)], tau=tau)[0]
        st = ref["states"]["r0"]
        if k == 2:
            lam = np.stack([(st["sums"][:, j, 0] + st["sums"][:, j, 1]) / st["n"] for j in range(2)], axis=1)
        else:
            lam = ((st["sum_s"] + st["sum_c"]) / st["n"])[:, None]
        assert np.array_equal(rec["R"][:, g, :k], lam)
        assert np.array_equal(rec["R"][:, g, k + 7:], ref["x"])


def test_monitor_and_running_maxima(oracle):
    sys = StandardMap(6.0)
    rec = oracle.oracle_record(sys, _starts(32, 6), 1000, 1, QRSpectrum(MGS()), [100, 300, 600, 1000])
    R = rec["R"]
    det, symp, Mmax = R[:, :, 2], R[:, :, 3], R[:, :, 8]   # columns: l1, l2, det, symp, orth, sum, pair, G, M, x, p
    assert np.all(det <= 1e-13) and np.all(symp <= 1e-13) and np.all(Mmax >= 1)
    for c in (2, 3, 5, 6, 8):   # det, symp, sum, pair, M_max are running maxima
        assert np.all(np.diff(R[:, :, c], axis=1) >= 0)
    assert np.all(R[:, :, 5] <= 1e-12)      # lambda_1 + lambda_2 = 0 to rounding (eps_sum)


@pytest.mark.parametrize("L", [20, 100, 700])
def test_launch_windows_change_no_bit(oracle, L):
    sys = WrappedStandardMap(2.0)
    x0 = _starts(20, 7, True)
    a = oracle.oracle_record(sys, x0, 700, 10, QRSpectrum(HouseholderQR()), [50, 60, 300, 700])
    b = oracle.oracle_record(sys, x0, 700, 10, QRSpectrum(HouseholderQR()), [50, 60, 300, 700], launch_steps=L)
    for key in a:
        assert np.asarray(a[key]).tobytes() == np.asarray(b[key]).tobytes(), key


def test_shadow_rows_are_the_direct_runs_X2(oracle):
    """The two-trajectory records: row g holds X2 = sum / grid[g] of the same run to that step and its state."""
    sys = StandardMap(1.7)
    x0 = _starts(30, 8)
    grid = [10, 40, 100, 300]
    ends, R, fail = oracle.oracle_shadow(sys, x0, 300, d0=1e-8, tau=5, seed=4, grid=grid)
    assert (fail == 0).all()
    for g, N in enumerate(grid):
        e = oracle.oracle_shadow(sys, x0, N, d0=1e-8, tau=5, seed=4)
        assert np.array_equal(R[:, g, 0], (e["sum_s"] + e["sum_c"]) / N)
        assert np.array_equal(R[:, g, 8:], e["x"])
    e_all = oracle.oracle_shadow(sys, x0, 300, d0=1e-8, tau=5, seed=4)
    assert e_all.tobytes() == ends.tobytes()
