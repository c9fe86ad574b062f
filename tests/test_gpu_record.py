"""The study recorder on the B200 against the oracle, bit for bit: every row of R, the failing grid index, the
carried state, frame, estimator and monitor states, status and failing step, for the lifted and wrapped standard
maps and a linear map, Benettin and the five QR estimators, tau 1 and 5, in one launch and in windows."""
from __future__ import annotations

import numpy as np
import pytest

from chaos_b200 import (CGS, MGS, RGS, AugmentedQR, Benettin, HouseholderQR, LinearSymplecticMap, QRSpectrum,
                        StandardMap, WrappedStandardMap, record, torus_state)
from helpers import same_bits

pytestmark = pytest.mark.gpu

ESTS = [Benettin(), QRSpectrum(CGS()), QRSpectrum(MGS()), QRSpectrum(RGS()), QRSpectrum(HouseholderQR()),
        QRSpectrum(AugmentedQR())]


def _system(name):
    z = np.random.default_rng(31).uniform(0, 2 * np.pi, (200, 2))
    if name == "standard":
        return StandardMap(2.5), z
    if name == "wrapped":
        return WrappedStandardMap(6.0), np.array([torus_state(v) for v in z])
    return LinearSymplecticMap([[2.0, 1.0], [1.0, 1.0]]), z * 1e-6


def _words(a):
    """The 8-byte words of a record, every NaN pattern made one (NaN sign and payload are not IEEE-defined: the
    device's and the host CPU's arithmetic may differ there, as the other parity tests allow)."""
    w = np.ascontiguousarray(a).view(np.uint64).copy()
    f = w.view(np.float64)
    w[np.isnan(f)] = 0x7FF8000000000000
    return w


def _same(dev, ref):
    assert same_bits(dev.R, ref["R"]), "R"
    assert same_bits(dev.x, ref["x"]) and same_bits(dev.W, ref["W"]), "x / W"
    assert np.array_equal(_words(dev.states), _words(ref["states"])), "states"
    for key in ("fail", "code", "hstep"):
        assert np.array_equal(getattr(dev, key), ref[key]), key


@pytest.mark.parametrize("est", ESTS, ids=repr)
@pytest.mark.parametrize("name", ["standard", "wrapped", "linear"])
@pytest.mark.parametrize("tau", [1, 5])
def test_record_matches_oracle(oracle, est, name, tau):
    sys, x0 = _system(name)
    N = 300 if name != "linear" else 30
    grid = [g for g in (tau, 2 * tau, 10 * tau, 20 * tau, N) if g <= N]
    grid = sorted(set(grid))
    dev = record(sys, x0, N, tau, est, grid)
    ref = oracle.oracle_record(sys, x0, N, tau, est, grid)
    _same(dev, ref)


@pytest.mark.parametrize("L", [10, 60])
def test_record_windows(oracle, L):
    sys, x0 = _system("wrapped")
    grid = [5, 20, 40, 100, 240]
    dev = record(sys, x0, 240, 5, QRSpectrum(HouseholderQR()), grid, launch_steps=L)
    ref = oracle.oracle_record(sys, x0, 240, 5, QRSpectrum(HouseholderQR()), grid, launch_steps=L)
    _same(dev, ref)
    whole = record(sys, x0, 240, 5, QRSpectrum(HouseholderQR()), grid)
    assert whole.R.tobytes() == dev.R.tobytes()


def test_record_failures(oracle):
    """A non-finite start fails at the first segment (fail = 1); an overflowing orbit fails in a later segment; the
    rows before the failing one are kept, and everything equals the oracle."""
    sys, x0 = _system("standard")
    x = x0[:40].copy()
    x[3, 0] = np.nan
    x[9, 1] = 1e306
    grid = [1, 5, 50, 100]
    dev = record(sys, x, 100, 1, QRSpectrum(MGS()), grid)
    ref = oracle.oracle_record(sys, x, 100, 1, QRSpectrum(MGS()), grid)
    _same(dev, ref)
    assert dev.fail[3] == 1 and dev.fail[9] >= 1 and (np.delete(dev.fail, [3, 9]) == 0).all()


@pytest.mark.parametrize("name", ["standard", "wrapped"])
@pytest.mark.parametrize("L", [None, 40])
def test_shadow_record_matches_oracle(oracle, name, L):
    from chaos_b200 import record_shadow
    sys, x0 = _system(name)
    x0 = x0.copy()
    x0[5, 0] = np.nan            # fails at the start: the first segment
    grid = [5, 20, 100, 200]
    R, fail, ends = record_shadow(sys, x0, 200, 5, grid, d0=1e-8, seed=3, launch_steps=L)
    rends, rR, rfail = oracle.oracle_shadow(sys, x0, 200, d0=1e-8, tau=5, seed=3, grid=grid, launch_steps=L)
    assert same_bits(R, rR) and np.array_equal(fail, rfail)
    assert np.array_equal(_words(ends), _words(rends))
    assert fail[5] == 1


@pytest.mark.parametrize("name", ["wrapped", "standard"])
def test_record_mixed(name):
    """The mixed recorder (Float64 orbit, monitor and log sums, Float32 frame and QR): the orbit bit for bit the
    plain recorder's and every exponent row within 1e-3 of it."""
    sysm, x0 = _system(name)
    grid = np.array([10, 100, 1000, 5000])
    a = record(sysm, x0, 5000, 1, QRSpectrum(MGS()), grid)
    b = record(sysm, x0, 5000, 1, QRSpectrum(MGS()), grid, precision="mixed")
    assert same_bits(a.x, b.x)
    ok = (a.code == 0) & (b.code == 0)
    assert ok.mean() > 0.99
    assert np.max(np.abs(a.R[ok][:, :, :2] - b.R[ok][:, :, :2])) <= 1e-3


@pytest.mark.parametrize("name", ["standard", "wrapped"])
def test_record_to_run_store(oracle, tmp_path, name):
    """The device record of a chunk (some orbits failing) through the run store: the orbit records built from it
    equal, bit for bit, those built from the oracle's record, and the chunk file reads back bit for bit."""
    from types import SimpleNamespace

    from chaos_b200 import run_store as RS
    sys, x0 = _system(name)
    x = x0[:24].copy()
    x[3, 0] = np.nan
    grid = [5, 20, 100, 200]
    est = QRSpectrum(MGS())
    dev = record(sys, x, 200, 5, est, grid)
    ref = oracle.oracle_record(sys, x, 200, 5, est, grid)
    tol = {"det_residual_tol": 16.0, "pairing_residual_tol": 16.0, "orthogonality_tol": 16.0}
    items = [{"orbit": i + 1, "system": name, "param": "6.0", "x0": "x", "p0": "p", "design_class": "chaotic",
              "orbit_seed": str(i), "hash": "h%d" % i, "method": "L4", "horizon": 200, "tau": 5, "vectors": 2,
              "coordinate_mode": "wrapped" if name == "wrapped" else "lifted"} for i in range(len(x))]
    a = RS.orbit_records(dev, items, tol)
    b = RS.orbit_records(SimpleNamespace(R=ref["R"], grid=np.asarray(grid), fail=ref["fail"], k=2,
                                         states=ref["states"], code=ref["code"], hstep=ref["hstep"]), items, tol)
    assert all(RS.same_orbit(u, v) for u, v in zip(a, b))
    assert np.all(np.isnan(a[3].state)) and a[3].t.sum() == 0
    p = str(tmp_path / "chunk-00001.h5")
    RS.write_chunk(p, {"schema_version": 2, "backend": "gpu", "method": "L4"}, a)
    back = RS.read_chunk(p)
    assert back.attrs["complete"] is True and all(RS.same_orbit(u, v) for u, v in zip(a, back.orbits))
