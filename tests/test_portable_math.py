"""The oracle's portable transcendentals (the device kernels run the same operation sequences, bit for bit, as the
GPU parity tests show) against the host's libm: sin / cos and log within 1 ulp, exp within 1 ulp over the whole
range including the subnormal results, atan2 within 2 ulp with the C99 signed-zero and infinity cases."""
from __future__ import annotations

import math

import numpy as np


def _ulps(a, b):
    a, b = np.asarray(a), np.asarray(b)
    sp = np.spacing(np.maximum(np.abs(a), np.abs(b)))
    with np.errstate(invalid="ignore"):
        return np.where(a == b, 0.0, np.abs(a - b) / sp)


def _run(oracle, name, *args, mode=0):
    args = [np.ascontiguousarray(a, dtype=np.float64) for a in args]
    out = np.empty_like(args[0])
    getattr(oracle.lib(), name)(mode, *[oracle._dp(a) for a in args], oracle._dp(out), len(out))
    return out


def test_sincos_and_log(oracle):
    x = np.random.default_rng(1).uniform(-1e4, 1e4, 200_000)
    s = np.empty_like(x)
    c = np.empty_like(x)
    oracle.lib().oracle_sincos(0, oracle._dp(x), oracle._dp(s), oracle._dp(c), len(x))
    assert _ulps(s, np.sin(x)).max() <= 1 and _ulps(c, np.cos(x)).max() <= 1
    y = np.exp(np.random.default_rng(2).uniform(-700, 700, 200_000))
    assert _ulps(_run(oracle, "oracle_log", y), np.log(y)).max() <= 1


def test_exp(oracle):
    rng = np.random.default_rng(3)
    x = np.concatenate([rng.uniform(-745, 709.78, 300_000), rng.uniform(-1, 1, 100_000), rng.uniform(-745.2, -708, 50_000),
                        [0.0, -0.0, 1.0, -1.0, 709.782712893384, -745.1332191019411, 710.0, -746.0, np.inf, -np.inf]])
    got = _run(oracle, "oracle_exp", x)
    with np.errstate(over="ignore"):
        ref = np.exp(x)
    normal = np.abs(ref) >= np.finfo(np.float64).tiny
    assert _ulps(got[normal], ref[normal]).max() <= 1
    assert np.max(np.abs(got[~normal] - ref[~normal])) <= 5e-324        # subnormal results: within one unit of 2^-1074
    assert got[-4] == np.inf and got[-3] == 0.0 and got[-2] == np.inf and got[-1] == 0.0
    assert math.isnan(_run(oracle, "oracle_exp", [np.nan])[0])


def test_atan2(oracle):
    rng = np.random.default_rng(4)
    y = rng.standard_normal(300_000) * 10.0 ** rng.uniform(-5, 5, 300_000)
    x = rng.standard_normal(300_000) * 10.0 ** rng.uniform(-5, 5, 300_000)
    got = _run(oracle, "oracle_atan2", y, x)
    assert _ulps(got, np.arctan2(y, x)).max() <= 2
    special = [(0.0, 1.0), (-0.0, 1.0), (0.0, -1.0), (-0.0, -1.0), (0.0, 0.0), (-0.0, -0.0), (1.0, 0.0), (-1.0, -0.0),
               (np.inf, 1.0), (-np.inf, -1.0), (1.0, np.inf), (-1.0, -np.inf), (np.inf, np.inf), (-np.inf, -np.inf),
               (1e-300, 1e300), (1e300, 1e-300), (3.0, -4.0)]
    ys, xs = np.array([p[0] for p in special]), np.array([p[1] for p in special])
    g = _run(oracle, "oracle_atan2", ys, xs)
    r = np.arctan2(ys, xs)
    assert _ulps(g, r).max() <= 2 and np.array_equal(np.signbit(g), np.signbit(r))
