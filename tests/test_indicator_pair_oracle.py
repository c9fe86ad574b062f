"""The indicator recorder's pair kind on the oracle (CPU): the known answers of the reference's RLI tests
(test/rli/rl_ac01_03.jl:142-180: a constant tangent gives DL = RLI = 0 exactly with s_A = s_B bitwise; the K = 0 shear
with independent vectors gives DL_n = ln sqrt(n^2 + 1) / n), each column's log sum bitwise the single-orbit Benettin
sum (rli.jl:6-8), the chain statement, the pairing failure, the monitor on orbit A, windows, and pair_start's checks
(test/rli/rl_ac04_07.jl:144-246)."""
from __future__ import annotations

import math

import numpy as np
import pytest

from chaos_b200 import (Benettin, LinearSymplecticMap, NumericalHealthError, StandardMap, WrappedStandardMap,
                        pair_frame, pair_start, record_indicator_pairs, torus_state)
from chaos_b200.propagate import FrameSpec
from chaos_b200.reducers import RLI

CHAINS = [["RLI"], ["RLI", "MEGNO"], ["MEGNO", "RLI"]]


def _xis(n, seed):
    a = np.random.default_rng(seed).uniform(0, 2 * np.pi, n)
    return np.stack([np.cos(a), np.sin(a)], axis=1)


def _pairs(sys, x0s, xis, Dx):
    zs = [pair_start(sys, x, u, Dx, orbit=j + 1)[0] for j, (x, u) in enumerate(zip(x0s, xis))]
    return np.array(zs), np.array([pair_frame(u) for u in xis])


def _rli_state(rec, chain_bytes_before=0):
    dt = RLI().dtype(4, 2)
    return np.frombuffer(rec["states"][:, chain_bytes_before:chain_bytes_before + dt.itemsize].tobytes(), dtype=dt)


@pytest.mark.parametrize("Dx", [1e-12, 1e-6])
@pytest.mark.parametrize("tau", [1, 5])
def test_constant_tangent_gives_exactly_zero(oracle, Dx, tau):
    sys = LinearSymplecticMap([[2.0, 1.0], [1.0, 1.0]])
    xis = _xis(100, 2)
    z0, W0 = _pairs(sys, np.zeros((100, 2)), xis, Dx)
    grid = [n for n in (1, 10, 200) if n % tau == 0]
    rec = oracle.oracle_indicator_pairs(sys, z0, W0, 200, tau, ["RLI"], grid)
    assert (rec["fail"] == 0).all()
    assert np.all(rec["R"][:, :, 0] == 0) and np.all(rec["R"][:, :, 1] == 0)
    st = _rli_state(rec)
    assert np.array_equal(st["sA_s"], st["sB_s"]) and np.array_equal(st["sA_c"], st["sB_c"])


@pytest.mark.parametrize("wrapped", [False, True])
def test_zero_shear_gives_exactly_zero(oracle, wrapped):
    sys = WrappedStandardMap(0.0) if wrapped else StandardMap(0.0)
    z = np.random.default_rng(3).uniform(0, 2 * np.pi, (10, 2))
    x0s = z
    z0, W0 = _pairs(sys, x0s, _xis(10, 4), 1e-3)
    rec = oracle.oracle_indicator_pairs(sys, z0, W0, 1000, 1, ["RLI"], [10, 1000])
    assert np.all(rec["R"][:, :, :2] == 0)


def test_independent_vectors_on_the_shear(oracle):
    sys = StandardMap(0.0)
    z0 = np.array([[1.0, 2.0, 1.0 + 1e-3, 2.0]])
    W0 = np.array([[[1.0, 0.0], [0.0, 0.0], [0.0, 0.0], [0.0, 1.0]]])
    rec = oracle.oracle_indicator_pairs(sys, z0, W0, 100, 1, ["RLI"], [10, 100])
    for g, n in enumerate((10, 100)):
        dl = rec["R"][0, g, 0]
        assert dl > 0 and math.isclose(dl, math.log(math.sqrt(n * n + 1.0)) / n, rel_tol=1e-12)


@pytest.mark.parametrize("members", CHAINS, ids=",".join)
@pytest.mark.parametrize("name", ["standard", "wrapped"])
def test_log_sums_are_the_single_orbit_benettin_sums(oracle, members, name):
    sys = StandardMap(1.4) if name == "standard" else WrappedStandardMap(1.4)
    x0s = np.random.default_rng(5).uniform(0, 2 * np.pi, (20, 2))
    xis = _xis(20, 6)
    z0, W0 = _pairs(sys, x0s, xis, 1e-7)
    rec = oracle.oracle_indicator_pairs(sys, z0, W0, 300, 3, members, [3, 150, 300])
    off = 0 if members[0] == "RLI" else 200
    st = _rli_state(rec, off)
    s = sys.s
    for half, key in ((0, "sA"), (1, "sB")):
        ref = oracle.oracle_frames(sys, z0[:, half * s:(half + 1) * s], 300,
                                   [FrameSpec(1, (Benettin(),), xis[:, :, None].copy())], tau=3)[0]
        b = ref["states"]["r0"]
        assert np.array_equal(st[key + "_s"], b["sum_s"]) and np.array_equal(st[key + "_c"], b["sum_c"])
        assert np.array_equal(rec["x"][:, half * s:(half + 1) * s], ref["x"])


def test_chain_members_are_the_stand_alone_members(oracle):
    sys = StandardMap(2.2)
    z0, W0 = _pairs(sys, np.random.default_rng(7).uniform(0, 2 * np.pi, (16, 2)), _xis(16, 8), 1e-8)
    grid = [10, 100, 400]
    a = oracle.oracle_indicator_pairs(sys, z0, W0, 400, 2, ["RLI", "MEGNO"], grid)["R"]
    b = oracle.oracle_indicator_pairs(sys, z0, W0, 400, 2, ["MEGNO", "RLI"], grid)["R"]
    rli = oracle.oracle_indicator_pairs(sys, z0, W0, 400, 2, ["RLI"], grid)["R"]
    assert a[:, :, 0:2].tobytes() == rli[:, :, 0:2].tobytes()
    assert b[:, :, 6:8].tobytes() == rli[:, :, 0:2].tobytes()
    assert a[:, :, 2:8].tobytes() == b[:, :, 0:6].tobytes()


def test_pairing_failure(oracle):
    sys = StandardMap(1.0)
    z0, W0 = _pairs(sys, np.array([[0.3, 0.4], [1.0, 2.0]]), _xis(2, 9), 1e-6)
    W0[1, 2, 0] = 1e-3                              # an off-block entry in column 1
    rec = oracle.oracle_indicator_pairs(sys, z0, W0, 20, 2, ["RLI"], [2, 10, 20])
    assert rec["fail"].tolist() == [0, 1] and rec["code"].tolist() == [0, 3]
    st = _rli_state(rec)
    assert st["code"].tolist() == [0, 2] and st["column"][1] == 1 and st["value"][1] > 0
    assert np.all(rec["R"][1] == 0)
    err = RLI().error(st[1], 2, "cpu")
    assert err.what == "pairing"


def test_monitor_reads_orbit_a(oracle):
    sys = WrappedStandardMap(3.0)
    x0s = np.random.default_rng(10).uniform(0, 2 * np.pi, (12, 2))
    z0, W0 = _pairs(sys, x0s, _xis(12, 11), 1e-9)
    grid = [5, 50, 100]
    pr = oracle.oracle_indicator_pairs(sys, z0, W0, 100, 5, ["MEGNO", "RLI"], grid, ns=8)
    single = oracle.oracle_indicators(sys, z0[:, :4], 100, 5, ["SALI"], grid, ns=4)
    assert np.array_equal(pr["R"][:, :, 8:11], single["R"][:, :, 2:5])
    assert np.array_equal(pr["R"][:, :, 11:15], single["R"][:, :, 5:9])


@pytest.mark.parametrize("L", [4, 40])
def test_launch_windows_change_no_bit(oracle, L):
    sys = StandardMap(1.8)
    z0, W0 = _pairs(sys, np.random.default_rng(12).uniform(0, 2 * np.pi, (10, 2)), _xis(10, 13), 1e-5)
    a = oracle.oracle_indicator_pairs(sys, z0, W0, 120, 2, ["RLI", "MEGNO"], [2, 60, 120])
    b = oracle.oracle_indicator_pairs(sys, z0, W0, 120, 2, ["RLI", "MEGNO"], [2, 60, 120], launch_steps=L)
    for key in a:
        assert np.asarray(a[key]).tobytes() == np.asarray(b[key]).tobytes(), key


def test_pair_start_checks():
    sys = StandardMap(1.0)
    z, dx, dr, mode = pair_start(sys, [3.0, 1.0], [0.6, 0.8], 1e-12, orbit=1)
    assert mode == "lifted" and dx == 1e-12 and abs(dr - 1e-12) <= math.sqrt(2) * 2.2e-16 * 2 * math.pi
    with pytest.raises(NumericalHealthError) as e:          # a lifted gap of 2 pi reads as 0 (minimal image)
        pair_start(sys, [3.0, 1.0], [1.0, 0.0], 2 * math.pi, orbit=17)
    assert e.value.what == "separation" and e.value.orbit == 17 and e.value.value == 0.0
    with pytest.raises(NumericalHealthError):
        pair_start(sys, [3.0, 1.0], [1.0, 0.0], -1.0)
    w = WrappedStandardMap(1.0)
    z, dx, dr, mode = pair_start(w, [6.283185307179586 - 1e-13, 1.0], [1.0, 0.0], 1e-12)
    assert mode == "wrapped" and abs(dr - 1e-12) <= 4 * math.sqrt(2) * 2.2e-16 * 2 * math.pi
    assert np.array_equal(z[:4], torus_state([6.283185307179586 - 1e-13, 1.0]))


def test_pair_chain_outside_the_menu():
    sys = StandardMap(1.0)
    z0, W0 = _pairs(sys, np.array([[0.3, 0.4]]), _xis(1, 9), 1e-6)
    with pytest.raises(ValueError, match="outside the compiled menu"):
        record_indicator_pairs(sys, z0, W0, 10, 1, ["RLI", "RLI"], [10])
